// Test infrastructure: a C entry layer over the reference's OWN solver code.
//
// This file is compiled together with the reference sources where they lie
// (src/winds/Solver.cpp, Solver_CPU.cpp, Solver_CPU_RB.cpp, Wall.cpp,
// PolyBuilding.cpp and src/qes/Domain.cpp) by oracle/Makefile into
// oracle/_ref/libqesref.so.
// Nothing in the product links it; only tests/ and bench.py's CPU-baseline
// and reference legs load it, as the checker and the timed reference.
//
// Grid conventions follow qes::Domain (src/qes/Domain.cpp:7-31): the caller
// passes the base cell counts Nx, Ny, Nz; the staggered sizes are
// nx = Nx+1, ny = Ny+1, nz = Nz+2, cell arrays hold (nx-1)(ny-1)(nz-1) values
// and face arrays nx*ny*nz values. dz_array has nz-1 entries (ghost at 0).
#include <chrono>
#include <cstring>
#include <vector>

#include "qes/Domain.h"
#include "WINDSGeneralData.h"
#include "WINDSInputData.h"
#include "Solver_CPU.h"
#include "Solver_CPU_RB.h"
#include "Wall.h"
#include "RectangularBuilding.h"
#include "CutBuilding.h"
#include <iostream>

// The cut-cell rasterisation (src/winds/CutBuilding.cpp) needs the full
// WINDSGeneralData; PolyBuilding::setCellFlags calls it only for
// meshTypeFlag 1, which the oracle never sets. An empty definition stands in,
// as do the building parameterizations (upwind cavity, wakes, street canyon,
// side wall, rooftop, mixing: their own reference files), which PolyBuilding's
// virtual table names but the rasterisation never calls.
void CutBuilding::setCutCellFlags(WINDSGeneralData *, const PolyBuilding *, int) {}
void PolyBuilding::upwindCavity(const WINDSInputData *, WINDSGeneralData *) {}
void PolyBuilding::polygonWake(const WINDSInputData *, WINDSGeneralData *, int) {}
void PolyBuilding::streetCanyon(WINDSGeneralData *) {}
void PolyBuilding::streetCanyonModified(WINDSGeneralData *) {}
void PolyBuilding::sideWall(const WINDSInputData *, WINDSGeneralData *) {}
void PolyBuilding::rooftop(const WINDSInputData *, WINDSGeneralData *) {}
void PolyBuilding::NonLocalMixing(WINDSGeneralData *, TURBGeneralData *, int) {}

namespace {

// Domain with a caller-provided (possibly stretched) dz_array. The z and
// z_face arrays are rebuilt with the rules of Domain::defineVerticalGrid
// (src/qes/Domain.cpp:135-151). This must happen before a Solver is built,
// because Solver keeps its own copy of the Domain (src/winds/Solver.cpp:77-78).
qes::Domain make_domain(int Nx, int Ny, int Nz, float dx, float dy, const float *dz_array)
{
  float dzmin = dz_array[1];
  for (int k = 0; k < Nz + 1; ++k)
    if (dz_array[k] < dzmin) dzmin = dz_array[k];
  qes::Domain d(Nx, Ny, Nz, dx, dy, dzmin);
  const int nz = d.nz();
  d.dz_array.assign(dz_array, dz_array + (nz - 1));
  d.z_face.assign(nz, 0.0f);
  d.z_face[0] = -d.dz_array[0];
  d.z_face[1] = 0.0f;
  for (int k = 2; k < nz; ++k) d.z_face[k] = d.z_face[k - 1] + d.dz_array[k - 1];
  d.z.assign(nz - 1, 0.0f);
  d.z[0] = -0.5f * d.dz_array[0];
  for (int k = 1; k < nz - 1; ++k) d.z[k] = 0.5f * (d.z_face[k] + d.z_face[k + 1]);
  return d;
}

// Exposes the protected solve() and the lambda buffer of a reference solver.
template <class Base>
class Probe : public Base {
public:
  Probe(const qes::Domain &d, float tol) : Base(d, tol) {}
  void run(WINDSGeneralData *wgd, int itermax) { Base::solve(wgd, itermax); }
  std::vector<float> &lam() { return this->lambda; }
  std::vector<float> &lam_old() { return this->lambda_old; }
};

template <class S>
double run_solver(const qes::Domain &d, WINDSGeneralData &wgd, float tol, int itermax,
                  const float *lambda_init, float *lambda_out)
{
  Probe<S> solver(d, tol);
  if (lambda_init) {
    std::memcpy(solver.lam().data(), lambda_init, sizeof(float) * solver.lam().size());
    std::memcpy(solver.lam_old().data(), lambda_init, sizeof(float) * solver.lam().size());
  }
  auto t0 = std::chrono::steady_clock::now();
  solver.run(&wgd, itermax);
  auto t1 = std::chrono::steady_clock::now();
  if (lambda_out) std::memcpy(lambda_out, solver.lam().data(), sizeof(float) * solver.lam().size());
  return std::chrono::duration<double>(t1 - t0).count();
}

}  // namespace

extern "C" {

// OpenMP threads used by Solver_CPU_RB. Its convergence loop resets the shared
// max_error inside the parallel region (Solver_CPU_RB.cpp:166), so with more
// than one thread a run can stop early; parity runs use 1 thread, timing runs
// pass tol < 0 so the loop always runs to itermax.
void qesref_set_threads(int n) { omp_set_num_threads(n > 0 ? n : 1); }

// Wall::defineWalls + Wall::solverCoefficients (src/winds/Wall.cpp:44-350,
// 827-846) on a WINDSGeneralData built as allocateMemory leaves it
// (src/winds/WINDSGeneralData.cpp:1064-1121: e..n = 1, volume fractions 1).
// icellflag is read and written (defineWalls may rewrite flags).
int qesref_walls(int Nx, int Ny, int Nz, float dx, float dy, const float *dz_array,
                 int *icellflag, float *e, float *f, float *g, float *h, float *m, float *n)
{
  qes::Domain d = make_domain(Nx, Ny, Nz, dx, dy, dz_array);
  WINDSGeneralData wgd(d);
  const long nc = d.numCellCentered();
  for (auto *v : {&wgd.e, &wgd.f, &wgd.g, &wgd.h, &wgd.m, &wgd.n}) v->assign(nc, 1.0f);
  wgd.building_volume_frac.assign(nc, 1.0f);
  wgd.icellflag.assign(icellflag, icellflag + nc);
  Wall wall;
  wall.defineWalls(&wgd);
  wall.solverCoefficients(&wgd);
  std::memcpy(icellflag, wgd.icellflag.data(), sizeof(int) * nc);
  float *outs[6] = {e, f, g, h, m, n};
  std::vector<float> *ins[6] = {&wgd.e, &wgd.f, &wgd.g, &wgd.h, &wgd.m, &wgd.n};
  for (int q = 0; q < 6; ++q) std::memcpy(outs[q], ins[q]->data(), sizeof(float) * nc);
  return 0;
}

// Wall::setVelocityZero (src/winds/Wall.cpp:805-825) on u0, v0, w0 in place.
int qesref_set_velocity_zero(int Nx, int Ny, int Nz, float dx, float dy, const float *dz_array,
                             const int *icellflag, float *u0, float *v0, float *w0)
{
  qes::Domain d = make_domain(Nx, Ny, Nz, dx, dy, dz_array);
  WINDSGeneralData wgd(d);
  const long nc = d.numCellCentered(), nf = d.numFaceCentered();
  wgd.icellflag.assign(icellflag, icellflag + nc);
  wgd.u0.assign(u0, u0 + nf);
  wgd.v0.assign(v0, v0 + nf);
  wgd.w0.assign(w0, w0 + nf);
  Wall wall;
  wall.setVelocityZero(&wgd);
  std::memcpy(u0, wgd.u0.data(), sizeof(float) * nf);
  std::memcpy(v0, wgd.v0.data(), sizeof(float) * nf);
  std::memcpy(w0, wgd.w0.data(), sizeof(float) * nf);
  return 0;
}

// Wall::defineWalls, then the reference's own Wall::wallLogBC(WGD, true)
// (src/winds/Wall.cpp:352-803) on u0, v0, w0 in place, with WGD->z0 = z0, as
// qesWindsMain.cpp:157-166 runs it after a solve (u0 <- u first). The domain is
// make_domain's, so getDomainSize() gives (dx, dx, min dz). icellflag receives
// the flags after defineWalls.
int qesref_wall_log_bc(int Nx, int Ny, int Nz, float dx, float dy, const float *dz_array, int *icellflag,
                       float z0, float *u0, float *v0, float *w0)
{
  qes::Domain d = make_domain(Nx, Ny, Nz, dx, dy, dz_array);
  WINDSGeneralData wgd(d);
  const long nc = d.numCellCentered(), nf = d.numFaceCentered();
  for (auto *v : {&wgd.e, &wgd.f, &wgd.g, &wgd.h, &wgd.m, &wgd.n}) v->assign(nc, 1.0f);
  wgd.building_volume_frac.assign(nc, 1.0f);
  for (auto *v : {&wgd.ni, &wgd.nj, &wgd.nk, &wgd.ti, &wgd.tj, &wgd.tk, &wgd.wall_distance}) v->assign(nc, 0.0f);
  wgd.center_id.assign(nc, 0);
  wgd.icellflag.assign(icellflag, icellflag + nc);
  Wall wall;
  wall.defineWalls(&wgd);
  wgd.z0 = z0;
  wgd.u0.assign(u0, u0 + nf);
  wgd.v0.assign(v0, v0 + nf);
  wgd.w0.assign(w0, w0 + nf);
  {
    std::streambuf *keep = std::cout.rdbuf(nullptr);  // wallLogBC prints progress
    wall.wallLogBC(&wgd, true);
    std::cout.rdbuf(keep);
  }
  std::memcpy(icellflag, wgd.icellflag.data(), sizeof(int) * nc);
  std::memcpy(u0, wgd.u0.data(), sizeof(float) * nf);
  std::memcpy(v0, wgd.v0.data(), sizeof(float) * nf);
  std::memcpy(w0, wgd.w0.data(), sizeof(float) * nf);
  return 0;
}

// One call of the reference Solver::solve. kind 0 = Solver_CPU (serial,
// lexicographic, src/winds/Solver_CPU.cpp:42-238); kind 1 = Solver_CPU_RB
// (OpenMP red-black, src/winds/Solver_CPU_RB.cpp:41-291). lambda_init and
// lambda_out may be null. Returns the wall time of solve() in seconds.
double qesref_solve(int kind, int Nx, int Ny, int Nz, float dx, float dy, const float *dz_array,
                    const float *e, const float *f, const float *g, const float *h, const float *m,
                    const float *n, const int *icellflag, const float *u0, const float *v0,
                    const float *w0, float tol, int itermax, const float *lambda_init, float *u,
                    float *v, float *w, float *lambda_out)
{
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
  double t = kind == 0 ? run_solver<Solver_CPU>(d, wgd, tol, itermax, lambda_init, lambda_out)
                       : run_solver<Solver_CPU_RB>(d, wgd, tol, itermax, lambda_init, lambda_out);
  std::memcpy(u, wgd.u.data(), sizeof(float) * nf);
  std::memcpy(v, wgd.v.data(), sizeof(float) * nf);
  std::memcpy(w, wgd.w.data(), sizeof(float) * nf);
  return t;
}

// The reference's rectangular buildings on a cell-flag field: for each of the
// nb buildings b[q] = (x_start, y_start, length, width, height, base height),
// rotation 0, RectangularBuilding::parseValues builds its polygon
// (src/winds/RectangularBuilding.h:62-112), then PolyBuilding::setPolyBuilding
// and setCellFlags (src/winds/PolyBuilding.cpp:72-236) rasterise it with the
// stair-step method, in building order. icellflag (cell layout) is the
// field before the buildings on entry and after them on return;
// ibuilding_flag (nullable) receives each cell's building index, -1 elsewhere.
int qr_rect_building_flags(int Nx, int Ny, int Nz, float dx, float dy, const float *dz_array, int nb,
                           const float *b, int *icellflag, int *ibuilding_flag)
{
  qes::Domain d = make_domain(Nx, Ny, Nz, dx, dy, dz_array);
  WINDSGeneralData wgd(d);
  const size_t nc = (size_t)(d.nx() - 1) * (d.ny() - 1) * (d.nz() - 1);
  wgd.icellflag.assign(icellflag, icellflag + nc);
  wgd.ibuilding_flag.assign(nc, -1);
  wgd.icellflag_footprint.assign((size_t)(d.nx() - 1) * (d.ny() - 1), 1);
  ShimSimParams sp;
  WINDSInputData wid;
  wid.simParams = &sp;
  for (int q = 0; q < nb; ++q) {
    const float *B = b + 6 * q;
    auto &v = ParseInterface::shimValues();
    v.clear();
    v["xStart"] = B[0];
    v["yStart"] = B[1];
    v["length"] = B[2];
    v["width"] = B[3];
    v["height"] = B[4];
    v["baseHeight"] = B[5];
    v["buildingRotation"] = 0.0;
    RectangularBuilding rb;
    rb.parseValues();
    rb.setPolyBuilding(&wgd);
    rb.setCellFlags(&wid, &wgd, q);
  }
  std::memcpy(icellflag, wgd.icellflag.data(), sizeof(int) * nc);
  if (ibuilding_flag) std::memcpy(ibuilding_flag, wgd.ibuilding_flag.data(), sizeof(int) * nc);
  return 0;
}

}  // extern "C"
