// ORACLE — test infrastructure only.  Pieces shared by the two harnesses
// that run Apollo's compiled code (ref_limiter.cpp, ref_driver.cpp): the
// members of ApSolver that subsolvers reach through getParent(), and the
// grid boundary-condition plugins by their registered kind names
// (aphyperapps_register.cc).  Include once per library.
#ifndef APOLLO_ORACLE_REF_HARNESS_H
#define APOLLO_ORACLE_REF_HARNESS_H
#include <string>
#include <utility>
#include <vector>

#include <apsolver.h>
#include <wxexcept.h>
#include <wxgridbc.h>
#include "advection/wxgridfixedbc.h"
#include "euler/wxeulerdirichletbc.h"
#include "euler/wxeulerinflowbc.h"
#include "euler/wxeulerwallbc.h"
#include "euler/wxeulerzerogradientbc.h"
#include "euler/wxisentropicvortexbc.h"
#include "maxwell/wxmaxwelltranversemagneticbc.h"
#include "maxwell/wxphmaxwellconductingwallbc.h"

// --------------------------------------------------------------- solver ----
// Boundary conditions created by this harness, handed to the solver by init().
namespace {
std::vector<std::pair<std::string, ApSubSolver<double>*> > g_pending;
}

template <typename REAL>
ApSolver<REAL>::ApSolver(const std::string& name) : WxSolverBase<REAL>(name), tssolver(nullptr) {}
template <typename REAL>
ApSolver<REAL>::~ApSolver() {
  for (typename SubSolverMap_t::iterator i = _subSolvers.begin(); i != _subSolvers.end(); ++i) delete i->second;
}
template <typename REAL>
void ApSolver<REAL>::setup(const WxCryptSet&) {}
template <typename REAL>
void ApSolver<REAL>::init() {}
template <>
void ApSolver<double>::init() {
  for (size_t i = 0; i < g_pending.size(); ++i) _subSolvers[g_pending[i].first] = g_pending[i].second;
  g_pending.clear();
}
template <typename REAL>
void ApSolver<REAL>::solve() {}
template <typename REAL>
WxStepperStatus<REAL> ApSolver<REAL>::step(REAL, REAL, Vec, Vec) {
  return WxStepperStatus<REAL>();
}
template <typename REAL>
ApSubSolver<REAL>* ApSolver<REAL>::getSubSolver(const std::string& name) {
  typename SubSolverMap_t::iterator i = _subSolvers.find(name);
  if (i != _subSolvers.end()) return i->second;
  WxExcept wxe;
  wxe << "WxSolver::getSubSolver : SubSolver " << name << " not found";
  throw wxe;
}
template class ApSolver<float>;
template class ApSolver<double>;

namespace {
ApSubSolver<double>* make_bc(const std::string& kind) {
  if (kind == "gridFixedBC") return new WxGridFixedBC<double>();
  if (kind == "isentropicVortexBC") return new WxIsentropicVortexBC<double>();
  if (kind == "eulerWallBC") return new WxEulerWallBC<double>();
  if (kind == "eulerInflowBC") return new WxEulerInflowBC<double>();
  if (kind == "eulerZeroGradientBC") return new WxEulerZeroGradientBC<double>();
  if (kind == "eulerDirichletBC") return new WxEulerDirichletBC<double>();
  if (kind == "maxwellTransverseMagneticBC") return new WxMaxwellTransverseMagnetic<double>();
  if (kind == "phmConductingWallBC") return new WxPHMaxwellConductingWallBC<double>();
  return nullptr;
}
}  // namespace
#endif
