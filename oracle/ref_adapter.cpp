// ORACLE — test infrastructure only.  A thin C interface over Apollo's own
// equation-plugin classes, which oracle/Makefile compiles unmodified from the
// Apollo source tree into oracle/_ref/libapollo_ref.so.  Tests use it to check
// the restated per-point physics (flux, numerical flux, Riemann wave speeds,
// exprFunc initial conditions) against the reference code itself, and can plug
// it into the oracle's RHS loop (orc_set_ref_plugins).
//
// Bound reference interfaces:
//   WxHyperbolicEqnSet<double>::setup/flux/DGnumericalFlux/riemann
//     (src/hyper/wxhyperboliceqnset.cc:43-89, 163-204, 295-328)
//   WxExprFunc::setup/func (src/lib/wxexprfunction.cc:4-59)
//   WxHyperbolicSrcSet<double>::setup/sourceTerms (src/hyper/wxhyperbolicsrcset.cc:16-71)
//     with the tranverseMagneticSrc and pointCurrentSrc plugins
//     (src/hyperapps/maxwell/wxtransversemagneticsrc.h, wxpointcurrent.h)
#include <sstream>
#include <string>
#include <vector>
#include <cstring>

#include <wxcreator.h>
#include <wxcryptset.h>
#include <wxexcept.h>
#include <wxhyperboliceqnset.h>
#include <wxexprfunction.h>
#include "advection/wxadvectioneqn.h"
#include "euler/wxeulereqn.h"
#include "maxwell/wxphmaxwelleqn.h"
#include <wxhyperbolicsrcset.h>
#include "maxwell/wxtransversemagneticsrc.h"
#include "maxwell/wxpointcurrent.h"

// Registration of the three equation kinds under their Apollo names, as
// src/hyperapps/aphyperapps_register.cc does for the full build.
static WxCreator<WxAdvectionEqn<double>, WxHyperbolicEqn<double> > reg_adv("advectionEqn");
static WxCreator<WxEulerEqn<double>, WxHyperbolicEqn<double> > reg_euler("eulerEqn");
static WxCreator<WxPHMaxwellEqn<double>, WxHyperbolicEqn<double> > reg_maxwell("phMaxwellEqn");
// and the two closed-form source kinds (aphyperapps_register.cc:113-118)
static WxCreator<WxTransverseMagneticSrc<double>, WxHyperbolicSrc<double> > reg_tmsrc("tranverseMagneticSrc");
static WxCreator<WxpointCurrentSrc<double>, WxHyperbolicSrc<double> > reg_pcsrc("pointCurrentSrc");

namespace {
struct RefEqn {
  WxHyperbolicEqnSet<double> set;
  std::vector<double> df, amdq, apdq, sx, sy;
  double** wave = nullptr;
  unsigned meqn = 0, mwave = 0;
};
std::string g_err;
}

extern "C" {

const char* ref_last_error() { return g_err.c_str(); }

// text: a cryptset with one top-level set holding `Equations = [name]` and the
// equation's own set, exactly as in an Apollo input file.
void* ref_eqn_create(const char* text) {
  try {
    std::istringstream in(text);
    WxCryptSet wxc(in);
    RefEqn* r = new RefEqn();
    unsigned dirs[3] = {0, 1, 2};
    r->set.setDirs(dirs);
    r->set.setDim(2);
    r->set.setup(wxc);
    r->meqn = r->set.totalEqns();
    r->mwave = r->set.totalWaves();
    r->df.assign(r->meqn, 0.0); r->amdq.assign(r->meqn, 0.0); r->apdq.assign(r->meqn, 0.0);
    r->sx.assign(r->mwave, 0.0); r->sy.assign(r->mwave, 0.0);
    r->wave = new double*[r->meqn];
    for (unsigned i = 0; i < r->meqn; ++i) r->wave[i] = new double[r->mwave];
    return r;
  } catch (WxExcept& e) {
    g_err = "WxExcept";
    return nullptr;
  } catch (...) {
    g_err = "unknown exception";
    return nullptr;
  }
}

void ref_eqn_destroy(void* h) {
  RefEqn* r = (RefEqn*)h;
  for (unsigned i = 0; i < r->meqn; ++i) delete[] r->wave[i];
  delete[] r->wave;
  delete r;
}

int ref_eqn_meqn(void* h) { return (int)((RefEqn*)h)->meqn; }
int ref_eqn_mwave(void* h) { return (int)((RefEqn*)h)->mwave; }

void ref_flux(void* h, int d, const double* q, double* f) {
  RefEqn* r = (RefEqn*)h;
  double qq[16], x[5] = {0, 0, 0, 0, 0};
  std::memcpy(qq, q, r->meqn * sizeof(double));
  r->set.flux((unsigned)d, x, qq, nullptr, f);
}

// qM and qP are passed through mutable, as the reference may clamp them.
void ref_numflux(void* h, const double* n, double* qM, double* qP, double* f, double* lam) {
  RefEqn* r = (RefEqn*)h;
  double nn[2] = {n[0], n[1]};
  r->set.DGnumericalFlux(nn, qM, qP, f, lam);
}

// The equation set's primitive variables (WxHyperbolicEqnSet::getPrimitiveVariable);
// qc is mutable because Apollo's Euler floors rewrite it.
void ref_primitive(void* h, double* qc, double* qp) {
  RefEqn* r = (RefEqn*)h;
  r->set.getPrimitiveVariable(qc, qp);
}

// One node of the Tu-Aliabadi reconstruction (WxHyperbolicEqnSet::tuAndAliabadiLimiter).
void ref_ta_limit(void* h, double* avg_cons, double* avg_prim, double* dgrads, double* out) {
  RefEqn* r = (RefEqn*)h;
  r->set.tuAndAliabadiLimiter(avg_cons, avg_prim, dgrads, out);
}

// Wave speeds of the Riemann problem with ql = qr = q in x and y, reduced the
// way WxNodalDG2dMethod::init does (wxnodaldg2dmethod.cc:201-209): returns the
// max over waves of max(sx^2, sy^2).
double ref_speed2(void* h, const double* q) {
  RefEqn* r = (RefEqn*)h;
  double ql[16], qr[16], xc[4] = {0, 0, 0, 0};
  std::memcpy(ql, q, r->meqn * sizeof(double));
  std::memcpy(qr, q, r->meqn * sizeof(double));
  r->set.riemann(0, xc, xc, ql, qr, nullptr, nullptr, r->df.data(), r->wave, r->sx.data(), r->amdq.data(), r->apdq.data());
  r->set.riemann(1, xc, xc, ql, qr, nullptr, nullptr, r->df.data(), r->wave, r->sy.data(), r->amdq.data(), r->apdq.data());
  double lam = 0.0;
  for (unsigned mw = 0; mw < r->mwave; ++mw) {
    double a = r->sx[mw] * r->sx[mw], b = r->sy[mw] * r->sy[mw];
    double m1 = lam > a ? lam : a;
    lam = m1 > b ? m1 : b;
  }
  return lam;
}

// exprFunc initial condition from a cryptset holding the InitialCondition
// set's keys (exprList, progn and constants) under one top-level set.
void* ref_exprfunc_create(const char* text) {
  try {
    std::istringstream in(text);
    WxCryptSet wxc(in);
    WxExprFunc* f = new WxExprFunc();
    f->setup(wxc);
    return f;
  } catch (...) {
    g_err = "exprFunc setup failed";
    return nullptr;
  }
}

int ref_exprfunc_size(void* h) { return (int)((WxExprFunc*)h)->size(); }

void ref_exprfunc_eval(void* h, double t, double x, double y, double* out) {
  double txo[4] = {t, x, y, 0.0};
  ((WxExprFunc*)h)->func(3, txo, out);
}

void ref_exprfunc_destroy(void* h) { delete (WxExprFunc*)h; }

// Source set of `meqn` fields from a cryptset holding `Sources = [...]` and
// the sources' own sets under one top-level set.
void* ref_src_create(const char* text, int meqn) {
  try {
    std::istringstream in(text);
    WxCryptSet wxc(in);
    WxHyperbolicSrcSet<double>* s = new WxHyperbolicSrcSet<double>();
    s->setNumEqns((unsigned)meqn);
    s->setup(wxc);
    return s;
  } catch (...) {
    g_err = "source setup failed";
    return nullptr;
  }
}

// sourceTerms at tx = [t, x, y, 0, 0] for the state q (s receives meqn values).
void ref_src_eval(void* h, double t, double x, double y, double* q, double* s) {
  double tx[5] = {t, x, y, 0.0, 0.0};
  ((WxHyperbolicSrcSet<double>*)h)->sourceTerms(tx, q, nullptr, s);
}

void ref_src_destroy(void* h) { delete (WxHyperbolicSrcSet<double>*)h; }

}  // extern "C"
