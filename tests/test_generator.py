"""The city generator (qes-public_b200/csrc/qesb_city.cpp) against the
reference's wall routines (Wall.cpp:44-350, 805-846) and building rules."""
import numpy as np
import pytest

import qesb
from oracle import oracle as O


def test_walls_match_golden(golden):
    import os

    z = dict(np.load(os.path.join(os.path.dirname(__file__), "golden", "walls_city.npz")))
    d = qesb.Domain(int(z["Nx"]), int(z["Ny"]), int(z["Nz"]), 2.0, 2.0, 1.0, z["dz_array"])
    c = qesb.city_random(d, int(z["seed"]), 8, fp=(6, 20), h=(4, 30))
    w = qesb.city_build(d, c.buildings, c.inflow)
    np.testing.assert_array_equal(np.where(w.icellflag == 0, 0, w.icellflag), z["flag_in"])
    np.testing.assert_array_equal(w.icellflag, z["icellflag"])
    for k in "efghmn":
        np.testing.assert_array_equal(getattr(w, k), z[k])


@pytest.mark.skipif(not O.ref_available(), reason="reference build oracle/_ref absent")
@pytest.mark.parametrize("seed", [1, 2, 3])
def test_walls_and_solid_faces_match_reference(seed):
    d = qesb.Domain(36, 30, 18, 2.0, 2.0, 1.0, qesb.city_dz(18, 1.0, 1.03))
    c = qesb.city_random(d, seed, 7, fp=(6, 16), h=(4, 24))
    w = qesb.city_build(d, c.buildings, c.inflow)
    flag, *co = O.ref_walls(d, w.icellflag)
    np.testing.assert_array_equal(flag, w.icellflag)
    for a, b in zip(co, (w.e, w.f, w.g, w.h, w.m, w.n)):
        np.testing.assert_array_equal(a, b)
    # setVelocityZero applied to the generator's profile leaves it unchanged
    u0, v0, w0 = O.ref_set_velocity_zero(d, w.icellflag, w.u0, w.v0, w.w0)
    np.testing.assert_array_equal(u0, w.u0)
    np.testing.assert_array_equal(v0, w.v0)
    np.testing.assert_array_equal(w0, w.w0)


@pytest.mark.skipif(not O.ref_available(), reason="reference build oracle/_ref absent")
@pytest.mark.parametrize("nx,ny,nz,seed,nb", [(36, 30, 18, 1, 7), (64, 48, 24, 2, 12), (100, 90, 30, 3, 20),
                                              (128, 128, 64, 1001, 40)])
def test_building_rasterisation_matches_reference_polybuilding(nx, ny, nz, seed, nb):
    """The buildings' stair-step cells, from the product generator and from the
    oracle's restatement, against the reference's own RectangularBuilding /
    PolyBuilding code (PNPOLY cell-centre test, k range from z and z_face) run
    on the same field before the buildings (fluid 1, ground plane 2)."""
    from oracle import city as OC

    d = qesb.Domain(nx, ny, nz, 2.0, 2.0, 1.0, qesb.city_dz(nz, 1.0, 1.03))
    c = qesb.city_random(d, seed, nb, fp=(6, 16), h=(4, 24))
    w = qesb.city_build(d, c.buildings, c.inflow)
    b = np.array([[x.x_start, x.y_start, x.length, x.width, x.height, x.base_height] for x in c.buildings],
                 np.float32)
    assert len(b) > 0
    X, Y, Z = nx, ny, nz + 1
    before = np.ones((Z, Y, X), np.int32)
    before[0] = 2
    flag, ib = O.ref_rect_building_flags(d, b, before.ravel())
    np.testing.assert_array_equal(w.icellflag, flag)
    assert (ib[flag == 0] >= 0).all() and (ib[flag != 0] == -1).all()
    od = OC.Domain(nx, ny, nz, 2.0, 2.0, d.dz_array)
    np.testing.assert_array_equal(OC.city_flags(od, b), flag)


def test_cuboid100_cells():
    """20x20x20 m cuboid at x, y in [40, 60] m: PNPOLY on cell centres puts
    cells 40..59 inside; heights 0..20 m give k = 1..20 (z[k] = k - 0.5)."""
    w = qesb.cuboid100()
    d = w.domain
    f = w.icellflag.reshape(d.cell_shape())
    solid = np.argwhere(f[1:] == 0)
    assert solid[:, 0].min() + 1 == 1 and solid[:, 0].max() + 1 == 20
    assert solid[:, 1].min() == 40 and solid[:, 1].max() == 59
    assert solid[:, 2].min() == 40 and solid[:, 2].max() == 59
    assert (f[0] == 2).all()


def test_power_law_profile():
    w = qesb.cuboid100()
    d = w.domain
    u0 = w.u0.reshape(d.face_shape())
    for k in (1, 10, 30, 50):
        expect = np.float32(np.float32(1.0) * np.float32(5.0)) * np.float32(
            np.power(np.float32(d.z[k] / np.float32(10.0)), np.float32(0.15), dtype=np.float32))
        assert abs(float(u0[k, 5, 5]) - float(expect)) <= 2e-6 * float(expect)
    assert (w.v0 == 0).all() and (w.w0 == 0).all()
    assert (u0[0] == 0).all() and (u0[-1] == 0).all()


def test_random_city_is_seeded_and_non_overlapping():
    d = qesb.config_domain("city400")
    a = qesb.city_random(d, 42, 60)
    b = qesb.city_random(d, 42, 60)
    assert len(a.buildings) == 60
    assert [(x.x_start, x.y_start, x.length, x.width, x.height) for x in a.buildings] == \
           [(x.x_start, x.y_start, x.length, x.width, x.height) for x in b.buildings]
    for i, p in enumerate(a.buildings):
        assert 10 <= p.length <= 40 and 10 <= p.width <= 40 and 10 <= p.height <= 60
        for q in a.buildings[:i]:
            overlap = (p.x_start < q.x_start + q.length and q.x_start < p.x_start + p.length and
                       p.y_start < q.y_start + q.width and q.y_start < p.y_start + p.width)
            assert not overlap
    assert 3 <= a.inflow.u_ref <= 10 and 0.1 <= a.inflow.p <= 0.3 and 0 <= a.inflow.dir_deg < 360


def test_stretched_dz():
    dz = qesb.city_dz(100, 1.0, 1.03)
    assert dz[0] == dz[1] == 1.0
    assert abs(dz[100] - 1.03 ** 99) < 1e-3


def test_city_inflow_reuses_geometry():
    """qesb_city_inflow over a built city's flags gives the winds
    qesb_city_build gives for that inflow (flags and coefficients shared)."""
    w, c = qesb.random_city("city128", 5)
    same = qesb.city_inflow(w, c.inflow)
    for a, b in ((same.u0, w.u0), (same.v0, w.v0), (same.w0, w.w0)):
        np.testing.assert_array_equal(a, b)
    other = qesb.Inflow(c.inflow.u_ref, c.inflow.z_ref, c.inflow.p, (c.inflow.dir_deg + 130.0) % 360.0)
    ref = qesb.city_build(w.domain, c.buildings, other)
    got = qesb.city_inflow(w, other)
    for a, b in ((got.u0, ref.u0), (got.v0, ref.v0), (got.w0, ref.w0), (got.e, ref.e), (got.icellflag, ref.icellflag)):
        np.testing.assert_array_equal(a, b)


@pytest.mark.skipif(not O.ref_available(), reason="reference build oracle/_ref absent")
@pytest.mark.parametrize("name,seed", [("city128", 1001), ("city128", 1002), ("city256", 500000), ("city256", 500001)])
def test_reference_leg_cities_equal_the_product_generator(name, seed):
    """The benchmark's reference leg builds its cities without the product
    library (oracle/city.py: the layout, flags and inflow restated in C, the
    walls and solid faces by the reference's Wall.cpp); they must be the
    product generator's cities bit for bit."""
    from oracle import city as OC

    wr = OC.random_city(name, seed)
    wp, _ = qesb.random_city(name, seed)
    np.testing.assert_array_equal(wr.domain.dz_array, wp.domain.dz_array)
    for k in ("icellflag", "e", "f", "g", "h", "m", "n", "u0", "v0", "w0"):
        np.testing.assert_array_equal(getattr(wr, k), getattr(wp, k), err_msg=k)
