"""The persistent rung kernel (csrc/fvm_fused.cu): captured individual-timestep
steps that involve few cells run every stage from the slope limiter to the
reconstruction as one cooperative launch.  It calls the stage kernels' own
per-cell and per-face functions over the same lists, so its steps must give
the stage kernels' bits, and through them stay at parity with the reference."""
import numpy as np
import pytest

from common import GOLDEN_STEP_CASES, RTOL_FP64, golden_params, load_golden, setup_case
from test_gpu_parity import assert_state_close, gpu_system

pytestmark = pytest.mark.gpu


def same_bits(a, b):
    sa, sb = a.get_state(), b.get_state()
    for k in sa:
        assert np.array_equal(sa[k], sb[k]), k
    assert a.time == b.time and a.tsys_ticks == b.tsys_ticks


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_fused_steps_give_the_stage_kernels_bits(precision):
    """A blast with individual timesteps: eager stage-kernel steps against
    replayed steps with every partial step in the persistent kernel."""
    import fvmhd3d_b200 as F
    prec = F.FVM_PREC_FP32 if precision == "fp32" else F.FVM_PREC_FP64
    m, W = setup_case(16, "blast", seed=4, noise=0.02)
    a, b = gpu_system(m, W, precision=prec), gpu_system(m, W, precision=prec)
    b.set_fused(m.ncell - 1)
    counts = [a.step(shared=False) for _ in range(12)]
    cells, _ = b.run(12, shared=False)
    assert cells == sum(counts)
    partial = sum(1 for c in counts if c < m.ncell)
    assert partial >= 3 and b.fused_steps >= partial
    same_bits(a, b)


def test_fused_steps_with_adjust_replays_and_threshold():
    """A blast with a 1e6 pressure contrast (adjust_timesteps replays in
    several steps), the persistent kernel taking only the steps that involve
    at most a third of the cells: the same bits as eager steps."""
    m, W = setup_case(12, "blast", seed=9, noise=0.02)
    W = W.copy()
    r = np.linalg.norm(m.pos - 0.5, axis=1)
    W[r < 0.12, 4] *= 1e4
    a, b = gpu_system(m, W), gpu_system(m, W)
    b.set_fused(m.ncell // 3)
    dirty = 0
    for _ in range(12):
        a.step(shared=False)
        dirty += a.adjust_stats()[0] > 0
    b.run(12, shared=False)
    assert dirty >= 2 and b.fused_steps >= 1
    same_bits(a, b)


@pytest.mark.parametrize("name", [n for n in GOLDEN_STEP_CASES if "individual" in n])
def test_fused_steps_vs_reference_golden(name):
    """The reference's own individual-timestep runs (blast, Keplerian disk
    with a sink, moving and static generators), replayed with the persistent
    kernel on every partial step: state at 1e-12, integers exact."""
    m, z = load_golden(name)
    s = gpu_system(m, z["W"], bnd=z.get("bnd"), **golden_params(z))
    s.set_fused(m.ncell - 1)
    cells, _ = s.run(int(z["nsteps"]), shared=False)
    assert cells == int(np.sum(z["out_nactive"]))
    assert s.fused_steps >= 1
    ref = {k[4:]: z[k] for k in z if k.startswith("out_")}
    assert_state_close(s.get_state(), ref, h=(np.mean(m.volume)) ** (1.0 / 3.0),
                       dt=2.0 ** -float(ref["rung"].max()) * golden_params(z).get("dtmax", 1.0 / 64))
    assert s.time == float(z["out_time"])


def test_eager_fused_steps_give_the_stage_kernels_bits():
    """Eager steps take the persistent kernel too (the host reads the
    involved-cell count after the lists are built): the same bits as eager
    stage-kernel steps, on the Keplerian disk golden (moving generators)."""
    m, z = load_golden("ref_disk4k_individual.npz")
    a = gpu_system(m, z["W"], bnd=z.get("bnd"), **golden_params(z))
    b = gpu_system(m, z["W"], bnd=z.get("bnd"), **golden_params(z))
    b.set_fused(m.ncell - 1)
    for _ in range(int(z["nsteps"])):
        assert a.step(shared=False) == b.step(shared=False)
    assert b.fused_steps >= 1
    same_bits(a, b)


def test_fused_setting_rejects_bad_values_and_global_steps_ignore_it():
    import fvmhd3d_b200 as F
    m, W = setup_case(8, "alfven", seed=2, noise=0.0)
    a, b = gpu_system(m, W), gpu_system(m, W)
    with pytest.raises(F.FvmError):
        b.set_fused(-1)
    b.set_fused(m.ncell)
    a.run(3, shared=True)
    b.run(3, shared=True)
    assert b.fused_steps == 0
    same_bits(a, b)
