// Solver_B200 adaptor: the reference Solver interface over the C ABI of
// libqesb200.so (include/qesb.h). Errors follow the reference GPU solvers'
// behaviour (src/winds/Solver_GPU_GlobalMemory.cu:58-65): print and exit.
#include "Solver_B200.h"

#include <cstdio>
#include <cstdlib>
#include <iostream>

namespace {
void check(qesb_status s, const char *what)
{
  if (s != QESB_OK) {
    std::fprintf(stderr, "[Solver_B200] %s failed (status %d): %s\n", what, (int)s, qesb_last_error());
    std::exit(EXIT_FAILURE);
  }
}
}  // namespace

Solver_B200::Solver_B200(qes::Domain domain_in, const float &tolerance, int device)
  : Solver(std::move(domain_in), tolerance)
{
  std::cout << "-------------------------------------------------------------------" << std::endl;
  std::cout << "[Solver]\t Initializing B200 Solver (GPU, " << qesb_version() << ") ..." << std::endl;
  qesb_grid g;
  g.Nx = domain.nx() - 1;
  g.Ny = domain.ny() - 1;
  g.Nz = domain.nz() - 2;
  g.dx = domain.dx();
  g.dy = domain.dy();
  g.dz_array = domain.dz_array.data();
  check(qesb_create(&g, tol, device, &handle_), "qesb_create");
}

Solver_B200::~Solver_B200()
{
  if (handle_) qesb_destroy(handle_);
}

void Solver_B200::solve(WINDSGeneralData *WGD, const int &itermax)
{
  auto start = std::chrono::high_resolution_clock::now();
  std::cout << "[Solver]\t Running B200 Solver (GPU) ..." << std::endl;
  check(qesb_set_tolerance(handle_, tol), "qesb_set_tolerance");
  if (stair_)
    check(qesb_set_inputs_flags(handle_, WGD->icellflag.data(), WGD->u0.data(), WGD->v0.data(), WGD->w0.data()),
          "qesb_set_inputs_flags");
  else
    check(qesb_set_inputs(handle_, WGD->e.data(), WGD->f.data(), WGD->g.data(), WGD->h.data(),
                          WGD->m.data(), WGD->n.data(), WGD->icellflag.data(), WGD->u0.data(),
                          WGD->v0.data(), WGD->w0.data()),
          "qesb_set_inputs");
  bool from_zero = true;  // a solve from lambda = 0: the first, or the first after resetLambda
  for (float x : lambda)
    if (x != 0.0f) {
      from_zero = false;
      break;
    }
  if (net_ && from_zero) {
    std::cout << "[Solver]\t Learned warm start ..." << std::endl;
    check(qesb_warm_start(handle_, net_), "qesb_warm_start");
  } else {
    check(qesb_set_lambda(handle_, lambda.data()), "qesb_set_lambda");
  }
  qesb_stats st{};
  check(qesb_solve(handle_, itermax, WGD->u.data(), WGD->v.data(), WGD->w.data(), &st), "qesb_solve");
  check(qesb_get_lambda(handle_, lambda.data()), "qesb_get_lambda");
  check(qesb_get_divergence(handle_, R.data()), "qesb_get_divergence");
  lambda_old = lambda;
  printf("[Solver]\t Residual after %d itertations: %2.9f\n", st.iterations, st.residual);
  auto finish = std::chrono::high_resolution_clock::now();
  std::chrono::duration<float> elapsed = finish - start;
  std::cout << "\t\t elapsed time: " << elapsed.count() << " s\n";
}
