// Drop-in demonstration: drives the solver exactly as qesWinds does
// (qesWinds/qesWindsMain.cpp:134-169): SolverFactory::create(type, domain,
// tol) with the B200 type registered as INTEGRATION.md describes (type 5; the
// reference's own types keep their meaning, type 1 being Solver_CPU_RB in an
// OpenMP build), then resetLambda and solve through Solver*. Inputs come from
// the library's city generator; u, v, w and lambda are written to a binary
// file for comparison.
// With a weights file (type 5 only) every solve that starts from lambda = 0
// uses the learned warm start (Solver_B200::useLearnedStart).
//   solver_b200_demo <out.bin> <Nx> <Ny> <Nz> <seed> <nbuildings> <itermax> <tol> [calls] [type] [weights] [stair]
// With "stair" as the last argument (type 5) the solves upload only the flags and initial winds
// (Solver_B200::useStairStepInputs); a weights argument of "-" means no network.
#include <cstdio>
#include <cstring>
#include <cstdlib>
#include <vector>

#include "SolverFactory.h"
#include "WINDSGeneralData.h"

int main(int argc, char **argv)
{
  if (argc < 9) {
    std::fprintf(stderr, "usage: %s out.bin Nx Ny Nz seed nbuildings itermax tol [calls]\n", argv[0]);
    return 2;
  }
  const int Nx = std::atoi(argv[2]), Ny = std::atoi(argv[3]), Nz = std::atoi(argv[4]);
  const unsigned long long seed = std::strtoull(argv[5], nullptr, 10);
  const int nb = std::atoi(argv[6]), itermax = std::atoi(argv[7]);
  const float tol = std::strtof(argv[8], nullptr);
  const int calls = argc > 9 ? std::atoi(argv[9]) : 1;
  const int type = argc > 10 ? std::atoi(argv[10]) : B200_Type;

  std::vector<float> dz(Nz + 1);
  qesb_city_dz(Nz, 1.0f, 1.03f, dz.data());
  qes::Domain domain(Nx, Ny, Nz, 2.0f, 2.0f, 1.0f);
  domain.dz_array = dz;
  WINDSGeneralData wgd(domain);
  const long nc = domain.numCellCentered(), nf = domain.numFaceCentered();
  for (auto *v : {&wgd.e, &wgd.f, &wgd.g, &wgd.h, &wgd.m, &wgd.n}) v->assign(nc, 1.0f);
  wgd.icellflag.assign(nc, 1);
  for (auto *v : {&wgd.u0, &wgd.v0, &wgd.w0, &wgd.u, &wgd.v, &wgd.w}) v->assign(nf, 0.0f);
  qesb_grid g{Nx, Ny, Nz, 2.0f, 2.0f, dz.data()};
  std::vector<qesb_building> b(nb > 0 ? nb : 1);
  int nbo = 0;
  qesb_inflow in{};
  if (qesb_city_random(&g, seed, nb, 6.0f, 16.0f, 4.0f, 20.0f, b.data(), &nbo, &in) != QESB_OK ||
      qesb_city_build(&g, nbo, b.data(), &in, wgd.icellflag.data(), wgd.e.data(), wgd.f.data(),
                      wgd.g.data(), wgd.h.data(), wgd.m.data(), wgd.n.data(), wgd.u0.data(),
                      wgd.v0.data(), wgd.w0.data()) != QESB_OK) {
    std::fprintf(stderr, "city generator failed: %s\n", qesb_last_error());
    return 1;
  }

  Solver *solver = SolverFactory::create(type, wgd.domain, tol);
  qesb_warmnet *net = nullptr;
  if (argc > 12 && type == B200_Type && std::strcmp(argv[12], "stair") == 0)
    static_cast<Solver_B200 *>(solver)->useStairStepInputs(true);
  if (argc > 11 && type == B200_Type && std::strcmp(argv[11], "-") != 0) {
    if (qesb_warmnet_load(argv[11], 0, &net) != QESB_OK) {
      std::fprintf(stderr, "warm-start network: %s\n", qesb_last_error());
      return 1;
    }
    static_cast<Solver_B200 *>(solver)->useLearnedStart(net);
  }
  solver->resetLambda();
  for (int c = 0; c < calls; ++c) solver->solve(&wgd, itermax);

  struct LambdaOf : Solver {  // reads the base class's protected lambda for the dump
    static const std::vector<float> &get(Solver *s) { return s->*(&LambdaOf::lambda); }
  };
  FILE *fo = std::fopen(argv[1], "wb");
  if (!fo) return 1;
  std::fwrite(wgd.u.data(), sizeof(float), nf, fo);
  std::fwrite(wgd.v.data(), sizeof(float), nf, fo);
  std::fwrite(wgd.w.data(), sizeof(float), nf, fo);
  std::fwrite(LambdaOf::get(solver).data(), sizeof(float), nc, fo);
  std::fclose(fo);
  // Solver has no virtual destructor: delete through the type the factory made
  if (type == B200_Type) delete static_cast<Solver_B200 *>(solver);
  qesb_warmnet_destroy(net);
  return 0;
}
