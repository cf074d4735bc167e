"""Synthetic meshes: benchmark sizes, reverse Cuthill-McKee ordering,
geometry against the reference's compute_mesh_geometry, and the reference's
own mesh validation."""
import numpy as np
import pytest


def _faces(nx, ny, nz):
    hexes = nx * ny * nz
    fb = 2 * (nx * ny + ny * nz + nx * nz)
    fi = (6 * hexes - fb) // 2
    return hexes, fi, fb


def test_ramp_sizes(cb):
    m = cb.HostMesh(cb.cases.ramp().spec)
    assert (m.n_cells, m.n_inner, m.n_faces - m.n_inner) == (4096, 10048, 4480)


@pytest.mark.parametrize("scale", [8, 2])
def test_plate_sizes(cb, scale):
    case = cb.cases.plate(scale=scale)
    s = case.spec
    m = cb.HostMesh(s)
    n, fi, fb = _faces(s.nx, s.ny, s.nz)
    assert (m.n_cells, m.n_inner, m.n_faces - m.n_inner) == (n, fi, fb)


def test_plate_full_size_matches_benchmark(cb):
    m = cb.HostMesh(cb.cases.plate().spec)
    assert (m.n_cells, m.n_inner, m.n_faces - m.n_inner) == (1048576, 3100672, 90112)


def test_bump_tet_sizes(cb):
    s = cb.cases.bump(scale=8).spec
    m = cb.HostMesh(s)
    hexes, _, fbq = _faces(s.nx, s.ny, s.nz)
    fb = 2 * fbq
    fi = (4 * 6 * hexes - fb) // 2
    assert (m.n_cells, m.n_inner, m.n_faces - m.n_inner) == (6 * hexes, fi, fb)
    # full size formula: 160x80x80 -> 6,144,000 / 12,224,000 / 128,000
    assert 6 * 160 * 80 * 80 == 6144000
    assert 2 * 2 * (160 * 80 + 80 * 80 + 160 * 80) == 128000


def test_three_zone_face_order_and_orientation(cb):
    m = cb.HostMesh(cb.cases.plate(scale=8).spec)
    a = m.arrays()
    ni = m.n_inner
    own, nei, pat = a["face_owner"], a["face_neigh"], a["face_patch"]
    assert np.all(nei[:ni] >= 0) and np.all(nei[ni:] == -1)
    key = own[:ni].astype(np.int64) * m.n_cells + nei[:ni]
    assert np.all(np.diff(key) > 0)
    bkey = pat[ni:].astype(np.int64) * m.n_cells + own[ni:]
    assert np.all(np.diff(bkey) >= 0)
    d = np.stack([a["face_centroid_x"] - a["cell_centroid_x"][own], a["face_centroid_y"] - a["cell_centroid_y"][own],
                  a["face_centroid_z"] - a["cell_centroid_z"][own]])
    nrm = np.stack([a["face_normal_x"], a["face_normal_y"], a["face_normal_z"]])
    assert np.all((d * nrm).sum(0) > 0)


def test_rcm_reduces_bandwidth_and_is_seeded(cb):
    case = cb.cases.plate(scale=4)
    spec = case.spec
    m1 = cb.HostMesh(spec)
    a = m1.arrays()
    ni = m1.n_inner
    bw = np.abs(a["face_owner"][:ni] - a["face_neigh"][:ni]).max()
    spec.reorder_rcm = 0
    m2 = cb.HostMesh(spec)
    b = m2.arrays()
    bw_perm = np.abs(b["face_owner"][:ni] - b["face_neigh"][:ni]).max()
    assert bw < bw_perm / 10
    spec.reorder_rcm = 1
    m3 = cb.HostMesh(spec)
    assert np.array_equal(m3.arrays()["cell_nodes"], a["cell_nodes"])
    spec.seed += 1
    m4 = cb.HostMesh(spec)
    assert not np.array_equal(m4.arrays()["node_x"], a["node_x"])


@pytest.mark.parametrize("name", ["ramp", "plate", "bump"])
def test_geometry_matches_reference(cb, refh, name):
    case = {"ramp": lambda: cb.cases.ramp(), "plate": lambda: cb.cases.plate(scale=8),
            "bump": lambda: cb.cases.bump(scale=16)}[name]()
    m = cb.HostMesh(case.spec)
    a = m.arrays()
    cell, face = refh.compute_geometry(m)
    for k, key in enumerate(["cell_centroid_x", "cell_centroid_y", "cell_centroid_z", "cell_volume"]):
        ref = cell[k]
        assert np.abs(a[key] - ref).max() <= 1e-13 * np.abs(ref).max(), key
    for k, key in enumerate(["face_centroid_x", "face_centroid_y", "face_centroid_z", "face_normal_x",
                             "face_normal_y", "face_normal_z", "face_area"]):
        ref = face[k]
        assert np.abs(a[key] - ref).max() <= 1e-13 * max(np.abs(ref).max(), 1.0), key
    refh.validate(m)  # the reference audit (aborts the process on a violation)


def test_connectivity_matches_reference(cb, refh):
    """The reference's aux connectivity on our mesh equals the stencils the
    oracle restatement builds (cell->faces, face and node neighbours)."""
    import port
    m = cb.HostMesh(cb.cases.bump(scale=16).spec)
    for kind in (0, 1, 2):
        off, val = refh.connectivity(m, kind)
        off2, val2 = port.connectivity(m, kind)
        assert np.array_equal(off, off2) and np.array_equal(val, val2), kind


def _geom(view, n, nf):
    def arr(k, m):
        return np.ctypeslib.as_array(getattr(view, k), shape=(m,)).copy()
    cells = {k: arr(k, n) for k in ("cell_volume", "cell_centroid_x", "cell_centroid_y", "cell_centroid_z")}
    faces = {k: arr(k, nf) for k in ("face_area", "face_centroid_x", "face_centroid_y", "face_centroid_z")}
    return cells, faces, arr("face_patch", nf)


@pytest.mark.parametrize("name", ["ramp", "plate", "bump", "sa_plate"])
def test_reference_pipeline_mesh_equals_generator(cb, refh, name):
    """The reference's own preprocessing (build_faces, migrate_local_mesh,
    compute_mesh_geometry, reorder_local_mesh(RCM), validate) on the cases'
    raw cells and nodes yields the mesh the product's generator builds: the
    same cells, faces and patches with the same geometry, up to the cell
    numbering.  The reference arm of the benchmark builds its meshes this way,
    without the product library."""
    case = cb.cases.ramp() if name == "ramp" else getattr(cb.cases, name)(scale=8)
    rm = refh.RefMesh(case.spec)
    hm = cb.HostMesh(case.spec)
    assert (rm.n_cells, rm.n_faces, rm.n_inner) == (hm.n_cells, hm.n_faces, hm.n_inner)
    assert rm.view.n_patches == hm.view.n_patches
    rc, rf, rp = _geom(rm.view, rm.n_cells, rm.n_faces)
    hc, hf, hp = _geom(hm.view, hm.n_cells, hm.n_faces)
    for k in rc:
        assert np.allclose(np.sort(rc[k]), np.sort(hc[k]), rtol=1e-13, atol=1e-13 * np.abs(hc[k]).max()), k
    for k in rf:
        assert np.allclose(np.sort(rf[k]), np.sort(hf[k]), rtol=1e-13, atol=1e-13 * np.abs(hf[k]).max()), k
    assert np.array_equal(np.bincount(rp[rp >= 0]), np.bincount(hp[hp >= 0]))
    # the same cells: centroid sets agree as a whole (lexicographic sort of
    # the centroids rounded well above the two codes' round-off)
    def order(c):
        key = [np.round(c[k] / 1e-9) for k in ("cell_centroid_z", "cell_centroid_y", "cell_centroid_x")]
        return np.lexsort(key)
    rk, hk = order(rc), order(hc)
    assert np.allclose(rc["cell_volume"][rk], hc["cell_volume"][hk], rtol=1e-12)
