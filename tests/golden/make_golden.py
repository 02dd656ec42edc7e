"""Generate the golden vectors in tests/golden/ from the reference's own code.

Run in a container that has the reference tree (oracle/Makefile builds
oracle/_ref/libqesref.so from it):

    python tests/golden/make_golden.py

Every output comes from the reference's compiled Solver_CPU / Solver_CPU_RB /
Wall code (oracle/_ref), never from this repository's solver. Inputs come
from the repository's city generator, whose coefficient arrays are replaced
here by the reference Wall routines' own output, so the fixtures pin both.

Files:
  walls_city.npz     icellflag before walls, and the reference's flags + e..n after
  small_cuboid.npz   inputs + Solver_CPU and Solver_CPU_RB results (u v w lambda), 200 iterations
  small_city.npz     same on a stretched grid with 5 buildings, 150 iterations
  cuboid100.npz      the 100x100x50 single-cuboid case: Solver_CPU run to itermax = 10000,
                     u v w lambda on a fixed stride subsample plus whole-field checksums
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "qes-public_b200"))
sys.path.insert(0, ROOT)

import qesb  # noqa: E402
from oracle import oracle as O  # noqa: E402

STRIDE = 7


def inputs_with_ref_walls(dom, wgd):
    flag0 = np.where(wgd.icellflag == 0, 0, wgd.icellflag).astype(np.int32)
    flag, e, f, g, h, m, n = O.ref_walls(dom, flag0)
    u0, v0, w0 = O.ref_set_velocity_zero(dom, flag, wgd.u0, wgd.v0, wgd.w0)
    wgd.icellflag, wgd.e, wgd.f, wgd.g, wgd.h, wgd.m, wgd.n = flag, e, f, g, h, m, n
    wgd.u0, wgd.v0, wgd.w0 = u0, v0, w0
    return wgd


def pack_inputs(dom, wgd):
    Nx, Ny, Nz = dom.base
    return dict(Nx=Nx, Ny=Ny, Nz=Nz, dx=dom.dx(), dy=dom.dy(), dz_array=dom.dz_array,
                icellflag=wgd.icellflag, e=wgd.e, f=wgd.f, g=wgd.g, h=wgd.h, m=wgd.m, n=wgd.n,
                u0=wgd.u0, v0=wgd.v0, w0=wgd.w0)


def solve_both(dom, wgd, itermax):
    out = {}
    for kind, tag in ((0, "cpu"), (1, "rb")):
        u, v, w, L, _ = O.ref_solve(dom, wgd, 1e-9, itermax, kind=kind)
        out.update({f"{tag}_u": u, f"{tag}_v": v, f"{tag}_w": w, f"{tag}_lambda": L})
    return out


def main():
    os.environ.setdefault("OMP_NUM_THREADS", "1")
    assert O.ref_available(), "build oracle/_ref first (make -C oracle)"

    # walls fixture
    d = qesb.Domain(48, 40, 24, 2.0, 2.0, 1.0, qesb.city_dz(24, 1.0, 1.03))
    c = qesb.city_random(d, 11, 8, fp=(6, 20), h=(4, 30))
    w = qesb.city_build(d, c.buildings, c.inflow)
    flag0 = np.where(w.icellflag == 0, 0, w.icellflag).astype(np.int32)
    flag, e, f, g, h, m, n = O.ref_walls(d, flag0)
    np.savez_compressed(os.path.join(HERE, "walls_city.npz"), Nx=48, Ny=40, Nz=24, dx=2.0, dy=2.0,
                        dz_array=d.dz_array, flag_in=flag0, icellflag=flag, e=e, f=f, g=g, h=h,
                        m=m, n=n, seed=11)

    # small cuboid (uniform grid)
    d = qesb.Domain(24, 20, 12, 1.0, 1.0, 1.0)
    w = qesb.city_build(d, [qesb.Building(8.0, 6.0, 6.0, 7.0, 6.0, 0.0)],
                        qesb.Inflow(5.0, 10.0, 0.15, 270.0))
    w = inputs_with_ref_walls(d, w)
    np.savez_compressed(os.path.join(HERE, "small_cuboid.npz"), itermax=200,
                        **pack_inputs(d, w), **solve_both(d, w, 200))

    # small city (stretched grid, oblique inflow)
    d = qesb.Domain(32, 28, 16, 2.0, 2.0, 1.0, qesb.city_dz(16, 1.0, 1.03))
    c = qesb.city_random(d, 5, 5, fp=(6, 14), h=(4, 16))
    w = qesb.city_build(d, c.buildings, c.inflow)
    w = inputs_with_ref_walls(d, w)
    np.savez_compressed(os.path.join(HERE, "small_city.npz"), itermax=150,
                        **pack_inputs(d, w), **solve_both(d, w, 150))

    # 100x100x50 cuboid, Solver_CPU to itermax = 10000 (the reference never
    # reaches tol = 1e-9 in FP32, so this is its full solve).
    w = qesb.cuboid100()
    d = w.domain
    w = inputs_with_ref_walls(d, w)
    u, v, ww, L, t = O.ref_solve(d, w, 1e-9, 10000, kind=0)
    sl = slice(0, None, STRIDE)
    np.savez_compressed(os.path.join(HERE, "cuboid100.npz"), stride=STRIDE, itermax=10000,
                        u=u[sl], v=v[sl], w=ww[sl], lam=L[sl],
                        u_sum=np.float64(u.astype(np.float64).sum()),
                        v_sum=np.float64(v.astype(np.float64).sum()),
                        w_sum=np.float64(ww.astype(np.float64).sum()),
                        max_div=O.max_divergence(d, w.icellflag, u, v, ww),
                        seconds=t)
    print("done; cuboid100 Solver_CPU seconds:", t)


if __name__ == "__main__":
    main()
