"""Snapshot format (the reference's system::dump_binary / read_binary) and
generator motion (orig_pos / orig_vel advanced by correct(), divBi).

CPU: the oracle's restatement of dump_binary reproduces the reference's own
snapshot files (committed in the golden fixtures) byte for byte, and the
reader parses them.  GPU: System.dump_binary through the C-ABI writes the
same header bytes and records equal to the reference's to float rounding of
values that agree to RTOL_FP64."""
import os

import numpy as np
import pytest

from common import GOLDEN_STEP_CASES, ORACLE_SO, RTOL_FP64, golden_params, load_golden, maxrel

from fvmhd3d_b200 import snapshot as S

needs_oracle = pytest.mark.skipif(not os.path.exists(ORACLE_SO), reason="oracle not built")


def run_oracle(name):
    from oracle.pyoracle import OracleSystem
    m, z = load_golden(name)
    o = OracleSystem(**golden_params(z))
    o.set_mesh(m)
    o.init_problem(z["W"], bnd=z.get("bnd"))
    for _ in range(int(z["nsteps"])):
        o.step(shared=bool(z["shared"]))
    return o, m, z


@needs_oracle
@pytest.mark.parametrize("name", GOLDEN_STEP_CASES)
def test_oracle_motion_and_dump_match_reference(name):
    o, m, z = run_oracle(name)
    mo = o.get_motion()
    for k in ("orig_pos", "orig_vel", "divb"):
        assert np.array_equal(mo[k], z["out_" + k]), k
    tsys, dt_global, iteration = o.clock()
    assert tsys == int(z["out_tsys"]) and iteration == int(z["nsteps"])
    assert o.dump_binary_bytes(bnd=z.get("bnd")) == z["out_dump_binary"].tobytes()


@pytest.mark.parametrize("name", GOLDEN_STEP_CASES)
def test_read_reference_snapshot(name):
    m, z = load_golden(name)
    hdr, rec = S.parse(z["out_dump_binary"].tobytes())
    n = m.ncell
    assert hdr["local_n"] == hdr["global_n"] == n and hdr["nproc"] == 1 and hdr["myproc"] == 0
    assert hdr["tsys"] == int(z["out_tsys"]) and hdr["iteration"] == int(z["nsteps"])
    assert hdr["t_global"] == np.float32(z["out_time"]) and hdr["periodic"] == -1
    assert np.array_equal(hdr["rmax"], np.asarray(m.box, np.float32))
    assert np.array_equal(rec["idx"], np.arange(n))
    assert np.array_equal(rec["pos"], z["out_orig_pos"].astype(np.float32))
    assert np.array_equal(rec["vel"], z["out_orig_vel"].astype(np.float32))
    assert np.array_equal(rec["volume"], m.volume.astype(np.float32))
    bnd = z.get("bnd", np.zeros(n, np.int32))
    assert np.array_equal(rec["boundary"], bnd)
    dens = z["out_U"][:, 0] / m.volume
    assert np.allclose(rec["dens"], dens, rtol=1e-6)
    dtmax = golden_params(z).get("dtmax", 1.0 / 64)
    assert np.array_equal(rec["dt"], (dtmax * 2.0 ** -z["out_rung"].astype(np.float64)).astype(np.float32))
    r = S.restart_inputs(hdr, rec, m.box)
    assert r["W"].shape == (n, 10) and r["tsys"] == hdr["tsys"]
    assert (r["pos"] >= 0).all() and (r["pos"] < np.asarray(m.box)).all()


def test_parse_rejects_damaged_files():
    _, z = load_golden("ref_alfven4_shared.npz")
    buf = bytearray(z["out_dump_binary"].tobytes())
    with pytest.raises(S.SnapshotError):
        S.parse(buf[:50])
    with pytest.raises(S.SnapshotError):
        S.parse(buf[:-4])
    bad = bytearray(buf)
    bad[S.HEADER_DTYPE.itemsize] = 7  # first record's leading marker
    with pytest.raises(S.SnapshotError):
        S.parse(bad)
    S.parse(buf)


def float_close(a, b, col_scale, rtol):
    """a, b float32 arrays: equal to one float rounding step of the larger
    magnitude, or within rtol of the column's largest magnitude."""
    a = a.astype(np.float64)
    b = b.astype(np.float64)
    ulp = np.spacing(np.maximum(np.abs(a), np.abs(b)).astype(np.float32)).astype(np.float64)
    return np.abs(a - b) <= np.maximum(ulp, rtol * col_scale)


@pytest.mark.gpu
@pytest.mark.parametrize("name", GOLDEN_STEP_CASES)
def test_gpu_motion_clock_and_dump_vs_reference(name, tmp_path):
    import fvmhd3d_b200 as F
    m, z = load_golden(name)
    s = F.System(**golden_params(z))
    s.set_mesh(m)
    s.init_problem(z["W"], bnd=z.get("bnd"))
    for _ in range(int(z["nsteps"])):
        s.step(shared=bool(z["shared"]))
    mo = s.get_motion()
    for k in ("orig_pos", "orig_vel"):
        assert maxrel(mo[k], z["out_" + k]).max() <= RTOL_FP64, k
    dscale = np.abs(z["out_divb"]).max()
    assert (np.abs(mo["divb"] - z["out_divb"]) <= np.maximum(
        np.spacing(np.abs(z["out_divb"])) * 2, 1e-10 * dscale)).all()
    tsys, dt_global, iteration = s.clock()
    assert tsys == int(z["out_tsys"]) and iteration == int(z["nsteps"])

    path = tmp_path / "snap.bin"
    s.dump_binary(path)
    got = path.read_bytes()
    ref = z["out_dump_binary"].tobytes()
    assert len(got) == len(ref)
    assert got[:S.HEADER_DTYPE.itemsize] == ref[:S.HEADER_DTYPE.itemsize]
    _, ra = S.parse(got)
    _, rb = S.parse(ref)
    for k in ("idx", "boundary", "dt", "volume", "J"):
        assert np.array_equal(ra[k], rb[k]), k
    for k in ("pos", "vel", "dens", "ethm", "pres", "velp", "B", "psi", "Ldivb", "entr"):
        a, b = ra[k], rb[k]
        scale = np.abs(b.astype(np.float64)).max(axis=0)
        assert float_close(a, b, scale, 1e-10).all(), k
