"""Host Voronoi builder: the reference's own mesh checks (closure
MPI/compute_update.cpp:307-320, total volume MPI/iterate.cpp:152-172, face
orientation asserts MPI/build_mesh_active.cpp:551-555)."""
import numpy as np
import pytest

import fvmhd3d_b200 as F


@pytest.mark.parametrize("nside", [4, 7, 12])
def test_volume_closure_orientation(nside):
    m = F.build_periodic(F.jittered_lattice(nside, 0.1, seed=nside), 1.0)
    assert abs(m.volume.sum() - 1.0) < 1e-12
    assert (m.volume > 0).all()
    assert m.closure_error().max() < 1e-10
    dri = m.centroid - m.pos[m.s1]
    assert np.abs(dri).max() < 0.5            # centroid in the frame of s1
    assert ((dri * m.n).sum(1) > 0).all()     # n points from s1 to s2
    off = m.cell_face_off
    assert off[0] == 0 and off[-1] == m.cell_face_ids.size
    # every face appears in the lists of both of its cells
    cnt = np.bincount(m.cell_face_ids, minlength=m.nface)
    assert (cnt == 2).all()
    cell_of_link = np.repeat(np.arange(m.ncell), np.diff(off))
    f = m.cell_face_ids
    assert ((m.s1[f] == cell_of_link) | (m.s2[f] == cell_of_link)).all()


def test_lattice_without_jitter_is_cubes():
    m = F.build_periodic(F.jittered_lattice(5, 0.0, seed=0), 1.0)
    areas = np.linalg.norm(m.n, axis=1)
    big = areas > 1e-8
    assert np.allclose(m.volume, 1.0 / 125)
    assert big.sum() == 3 * 125              # six faces per cube, shared
    assert np.allclose(areas[big], 1.0 / 25)


def test_deterministic():
    p = F.jittered_lattice(6, 0.1, seed=9)
    a = F.build_periodic(p, 1.0)
    b = F.build_periodic(p, 1.0, nthreads=1)
    assert np.array_equal(a.s1, b.s1) and np.array_equal(a.s2, b.s2)
    assert np.array_equal(a.n, b.n) and np.array_equal(a.cell_face_ids, b.cell_face_ids)
