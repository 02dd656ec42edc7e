// Solver_B200: the B200 lambda solve behind the reference's own Solver
// interface (src/winds/Solver.h:61-113), so it drops in beside Solver_CPU:
//
//     Solver *solver = new Solver_B200(WGD->domain, tol);   // or via SolverFactory type 5
//     solver->resetLambda();
//     solver->solve(WGD, itermax);
//
// Compiled inside the reference tree it includes the reference's Solver.h and
// WINDSGeneralData.h; it calls libqesb200.so only through include/qesb.h.
#pragma once

#include "Solver.h"
#include "qesb.h"

class Solver_B200 : public Solver
{
public:
  Solver_B200(qes::Domain domain_in, const float &tolerance, int device = 0);
  ~Solver_B200();

  Solver_B200(const Solver_B200 &) = delete;
  Solver_B200 &operator=(const Solver_B200 &) = delete;

  // The library handle, for the options the Solver interface has no place
  // for (qesb_set_prephase, qesb_set_option, qesb_set_stream, qesb_solve_batch).
  qesb_handle *handle() const { return handle_; }

  // The learned warm start (qesb_warm_start): every solve that would start
  // from lambda = 0 (the first one, and each one after resetLambda, as
  // qesWinds solves) starts from the network's prediction instead; a solve
  // that continues from a previous lambda (QES-Fire's repeated solves) keeps
  // it. The network is the caller's (qesb_warmnet_load); nullptr turns it off.
  void useLearnedStart(qesb_warmnet *net) { net_ = net; }

  // Stair-step inputs (qesb_set_inputs_flags): when the coefficients are the
  // ones Wall::solverCoefficients gives for the flags (meshTypeFlag 0, not read
  // from a file), each solve uploads only icellflag and u0, v0, w0 and the
  // library recomputes e..n from the flags on the device, bit for bit.
  void useStairStepInputs(bool on) { stair_ = on; }

protected:
  // Solver::solve semantics (src/winds/Solver_CPU.cpp:42-238): reads e..n,
  // icellflag, u0 v0 w0 and writes u v w of WGD. lambda lives in the base
  // class's vector between calls (uploaded before, downloaded after), so
  // Solver::resetLambda and the reference's cross-call warm start behave as
  // they do for Solver_CPU.
  virtual void solve(WINDSGeneralData *WGD, const int &itermax) override;

private:
  qesb_handle *handle_ = nullptr;
  qesb_warmnet *net_ = nullptr;
  bool stair_ = false;
};
