// Test/benchmark infrastructure: a C entry over the reference's own GPU
// solver, Solver_GPU_GlobalMemory (src/winds/Solver_GPU_GlobalMemory.cu),
// compiled from its sources by oracle/Makefile into oracle/_ref/libqesref_gpu.so.
// Used only as a timed comparator ("plain GPU SOR from lambda = 0" as the
// reference ships it); its results carry the reference GPU solvers' known
// defects (Neumann bound nx*ny, dy = dx), so they are not a parity target.
#include <chrono>
#include <cstring>
#include <vector>

#include "qes/Domain.h"
#include "WINDSGeneralData.h"
#include "Solver_GPU_GlobalMemory.h"

namespace {
qes::Domain make_domain(int Nx, int Ny, int Nz, float dx, float dy, const float *dz_array)
{
  float dzmin = dz_array[1];
  for (int k = 0; k < Nz + 1; ++k)
    if (dz_array[k] < dzmin) dzmin = dz_array[k];
  qes::Domain d(Nx, Ny, Nz, dx, dy, dzmin);
  d.dz_array.assign(dz_array, dz_array + (d.nz() - 1));
  return d;
}
}  // namespace

extern "C" double qesref_solve_gpu(int Nx, int Ny, int Nz, float dx, float dy, const float *dz_array,
                                   const float *e, const float *f, const float *g, const float *h,
                                   const float *m, const float *n, const int *icellflag, const float *u0,
                                   const float *v0, const float *w0, float tol, int itermax, float *u,
                                   float *v, float *w)
{
  // divergenceGlobal (Solver_GPU_GlobalMemory.cu:86) reads d_dz_array[k + 1]
  // for k = nz - 2, one float past its (nz - 1)-float allocation (:265). A
  // cudaMalloc'd block starts on a 256-byte boundary, so that float lies in
  // the same page as the block's last float unless (nz - 1) * 4 is a multiple
  // of 256; those grids are refused rather than run.
  if (((Nz + 1) * 4) % 256 == 0) return -1.0;
  qes::Domain d = make_domain(Nx, Ny, Nz, dx, dy, dz_array);
  WINDSGeneralData wgd(d);
  const long nc = d.numCellCentered(), nf = d.numFaceCentered();
  wgd.e.assign(e, e + nc);
  wgd.f.assign(f, f + nc);
  wgd.g.assign(g, g + nc);
  wgd.h.assign(h, h + nc);
  wgd.m.assign(m, m + nc);
  wgd.n.assign(n, n + nc);
  wgd.icellflag.assign(icellflag, icellflag + nc);
  wgd.u0.assign(u0, u0 + nf);
  wgd.v0.assign(v0, v0 + nf);
  wgd.w0.assign(w0, w0 + nf);
  wgd.u.assign(nf, 0.0f);
  wgd.v.assign(nf, 0.0f);
  wgd.w.assign(nf, 0.0f);
  struct Probe : Solver_GPU_GlobalMemory {
    Probe(const qes::Domain &dd, float t) : Solver_GPU_GlobalMemory(dd, t) {}
    void run(WINDSGeneralData *p, int it) { solve(p, it); }
  } solver(d, tol);
  auto t0 = std::chrono::steady_clock::now();
  solver.run(&wgd, itermax);
  auto t1 = std::chrono::steady_clock::now();
  std::memcpy(u, wgd.u.data(), sizeof(float) * nf);
  std::memcpy(v, wgd.v.data(), sizeof(float) * nf);
  std::memcpy(w, wgd.w.data(), sizeof(float) * nf);
  return std::chrono::duration<double>(t1 - t0).count();
}
