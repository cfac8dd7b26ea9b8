"""Bundles (bfpn_bundle_*): beams of one shape class advanced together with
one launch per operator per depth step.  Every beam's IDD history must equal
the same beam run alone through a single context, within 1e-6 of its peak
(mixed precision; the only difference allowed is the order of the IDD
partial sums), whether the beams join together or while others are running,
and whatever kernel variants the autotuner or the caller picks."""
import numpy as np
import pytest

from bfpn_gpu_b200 import Context, beams, capi

pytestmark = pytest.mark.gpu

TOL = 1e-6


def pick(ny, na, count, max_steps, seed=20261203):
    """`count` beams of the seeded uneven set (energy, material, sigma, Ng and
    depth as drawn) recast to one shape class, depth capped at max_steps."""
    pool = beams.uneven_beams(4 * count, seed=seed, ny_choices=(ny,), na_choices=(na,))
    out = []
    for r in pool[:count]:
        r.nsteps = min(r.nsteps, max_steps)
        out.append(r)
    return out


def alone(r):
    ctx = Context(r.cfg.grid(), r.cfg.phys(), capi.PREC_MIXED)
    ctx.load_tables(r.mu, r.sigma)
    ctx.init_beam()
    idd, proxy = ctx.step(r.nsteps)
    ctx.close()
    return idd, proxy


def check(got, ref):
    idd, _ = got
    ridd, _ = ref
    assert idd.shape == ridd.shape
    assert np.abs(ridd).max() > 0
    assert np.abs(idd - ridd).max() <= TOL * np.abs(ridd).max()


@pytest.mark.parametrize("ny,na", [(16, 12), (32, 16), (48, 20)])
def test_bundle_equals_beams_alone(ny, na):
    """Four beams (different energies, materials, Ng, sigma, depths) joining
    together; planes of 17, 33 and 49 points (whole-plane and row-streaming
    transport), 12, 16 and 20 angles per direction."""
    reqs = pick(ny, na, 4, 36)
    reqs[1].nsteps = 23  # slots finish at different steps
    refs = [alone(r) for r in reqs]
    with capi.Bundle(max_slots=8) as b:
        slots = [b.admit(r.beam()) for r in reqs]
        b.step(1000)
        assert b.running() == 0
        b.sync()
        assert "transport" in b.tuning()
        for s, ref in zip(slots, refs):
            check(b.collect(s), ref)


def test_bundle_continuous_admission():
    """Beams join while others run (first steps mixed with regular ones, a
    slot reused after its beam is collected)."""
    reqs = pick(16, 16, 5, 30, seed=7)
    refs = [alone(r) for r in reqs]
    got = {}
    with capi.Bundle(max_slots=3) as b:
        s0 = b.admit(reqs[0].beam())
        s1 = b.admit(reqs[1].beam())
        b.step(7)
        s2 = b.admit(reqs[2].beam())
        b.step(11)
        assert b.slot(s0)[0] == 18 and b.slot(s2)[0] == 11
        b.step(12)  # beams 0 and 1 finish (30 steps)
        got[0] = b.collect(s0)
        got[1] = b.collect(s1)
        s3 = b.admit(reqs[3].beam())
        s4 = b.admit(reqs[4].beam())
        assert {s3, s4} == {s0, s1}  # freed slots are reused
        b.step(1000)
        got[2] = b.collect(s2)
        got[3] = b.collect(s3)
        got[4] = b.collect(s4)
    for k, ref in enumerate(refs):
        check(got[k], ref)


def test_bundle_kernel_variants_agree():
    """Fixed variants (transport 8 / 16 angles per block, DST 2 / 3 stages,
    ring / register energy sweep) give the same IDD as the beam alone."""
    reqs = pick(20, 12, 2, 20, seed=11)
    refs = [alone(r) for r in reqs]
    for opts in ({capi.BUNDLE_OPT_TRANSPORT_ANGLES: 8, capi.BUNDLE_OPT_DST_STAGES: 3,
                  capi.BUNDLE_OPT_ENERGY_RING: 0},
                 {capi.BUNDLE_OPT_TRANSPORT_ANGLES: 16, capi.BUNDLE_OPT_DST_STAGES: 2,
                  capi.BUNDLE_OPT_ENERGY_RING: 1}):
        with capi.Bundle(max_slots=2) as b:
            for k, v in opts.items():
                b.set_option(k, v)
            slots = [b.admit(r.beam()) for r in reqs]
            b.step(100)
            for s, ref in zip(slots, refs):
                check(b.collect(s), ref)


def test_bundle_rejects_other_classes_and_bad_use():
    a = pick(16, 12, 1, 10)[0]
    other = pick(32, 12, 1, 10)[0]
    fp64 = pick(16, 12, 1, 10)[0]
    fp64.precision = capi.PREC_FP64
    with capi.Bundle(max_slots=1) as b:
        with pytest.raises(capi.BfpnError, match="mixed-precision"):
            b.admit(fp64.beam())
        s = b.admit(a.beam())
        with pytest.raises(capi.BfpnError, match="every slot is taken"):
            b.admit(a.beam())
        with pytest.raises(capi.BfpnError, match="steps left"):
            b.collect(s)
        b.step(3)
        assert b.slot(s) == (3, 10)
    with capi.Bundle(max_slots=2) as b:
        b.admit(a.beam())
        with pytest.raises(capi.BfpnError, match="shape class"):
            b.admit(other.beam())
