// ORACLE — test infrastructure only.  Runs Apollo's own limiters and grid
// boundary-condition plugins, compiled unmodified from the Apollo source tree
// by `oracle/Makefile reflim` into oracle/_ref/libapollo_reflim.so, so that
// tests can check the oracle's restatements against Apollo's code:
//   eulerLimiterHW                 src/hyperapps/euler/wxhesthavenwarburtoneulerlimiter.cc:62-485
//   tuAliabadiLimiter              src/hyperapps/multifluid/aptualiabadilimiter.cc:75-425
//     (with the eulerEqn and phMaxwellEqn plugins it takes its primitive
//     variables and reconstruction from)
//   gridFixedBC                    src/hyperapps/advection/wxgridfixedbc.cc
//   isentropicVortexBC             src/hyperapps/euler/wxisentropicvortexbc.cc
//   eulerWallBC, eulerInflowBC, eulerZeroGradientBC, eulerDirichletBC
//                                  src/hyperapps/euler/wxeuler*bc.cc
//   maxwellTransverseMagneticBC    src/hyperapps/maxwell/wxmaxwelltranversemagneticbc.cc
//   phmConductingWallBC            src/hyperapps/maxwell/wxphmaxwellconductingwallbc.cc
// with their bases (WxNodalDGLimiter, WxGridBC, ApSubSolver, WxStepper,
// WxSolverBase) also compiled unmodified.
//
// What this file supplies in place of PETSc and of Apollo's PETSc-bound code:
//   * the DM and Vec calls the limiter makes (declared in solver_stub/petsc.h),
//     over one array of K elements x Np nodes x the fields, with no ghost cells
//     (DMPlexGetHybridBounds returns K, where Apollo's ghost cells start);
//   * the out-of-line members of wxNodalDGgeometry2D that the limiter calls.
//     Apollo builds that object from a DMPlex with PETSc matrices
//     (wxnodaldggeometry2d.cc:18-135, 237-367), which cannot be compiled here;
//     the constructor below takes the node coordinates, face masks, mass matrix
//     and element-to-element-to-face table from the caller instead, and
//     Normals2d / GeometricFactors2d restate wxnodaldggeometry2d.cc:384-438.
//     The inline members (LimiterElementAVE, returnFmask, the accessors) are
//     Apollo's header code;
//   * the members of ApSolver that the limiter reaches through getParent()
//     (ref_harness.h): getSubSolver, the same lookup as apsolver.cc:160-169,
//     over the boundary conditions this harness registered;
//   * the PETSc vector norm that tuAliabadiLimiter's unused NaN check names.
#include <cmath>
#include <cstring>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include <wxcryptset.h>
#include <wxnodaldggeometry2d.h>
#include <wxnodaldglimiter.h>
#include "euler/wxhesthavenwarburtoneulerlimiter.h"
#include "multifluid/aptualiabadilimiter.h"
#include "ref_harness.h"
#include <wxcreator.h>
#include "advection/wxadvectioneqn.h"
#include "euler/wxeulereqn.h"
#include "maxwell/wxphmaxwelleqn.h"

// The equation kinds under their Apollo names, as aphyperapps_register.cc
// registers them, for tuAliabadiLimiter's equation set.
static WxCreator<WxAdvectionEqn<double>, WxHyperbolicEqn<double> > reg_adv("advectionEqn");
static WxCreator<WxEulerEqn<double>, WxHyperbolicEqn<double> > reg_euler("eulerEqn");
static WxCreator<WxPHMaxwellEqn<double>, WxHyperbolicEqn<double> > reg_maxwell("phMaxwellEqn");

// ---------------------------------------------------------------- DM, Vec ----
struct _p_DM {
  int K = 0, N = 0, Np = 0, dof = 0;  // dof per element: Np nodes x the fields
  std::vector<double> x, y, mass;      // [K][Np], [K][Np], [Np][Np]
  std::vector<int> conn, fmask;        // [K][6], [3 (N+1)]
};
struct _p_Vec {
  std::vector<double> a;
};

PetscErrorCode DMPlexGetHeightStratum(DM dm, PetscInt height, PetscInt* s, PetscInt* e) {
  *s = 0;
  *e = height == 0 ? dm->K : 0;
  return 0;
}
PetscErrorCode DMPlexGetHybridBounds(DM dm, PetscInt* cmax, PetscInt* fmax, PetscInt* e1, PetscInt* vmax) {
  if (cmax) *cmax = dm->K;
  if (fmax) *fmax = -1;
  if (e1) *e1 = -1;
  if (vmax) *vmax = -1;
  return 0;
}
PetscErrorCode DMPlexPointLocalRead(DM dm, PetscInt p, const PetscScalar* a, void* ptr) {
  *(const PetscScalar**)ptr = a + (size_t)p * dm->dof;
  return 0;
}
PetscErrorCode DMPlexPointLocalRef(DM dm, PetscInt p, PetscScalar* a, void* ptr) {
  *(PetscScalar**)ptr = a + (size_t)p * dm->dof;
  return 0;
}
PetscErrorCode DMGetLocalVector(DM dm, Vec* v) {
  *v = new _p_Vec();
  (*v)->a.assign((size_t)dm->K * dm->dof, 0.0);
  return 0;
}
PetscErrorCode DMRestoreLocalVector(DM, Vec* v) {
  delete *v;
  *v = nullptr;
  return 0;
}
PetscErrorCode DMGlobalToLocalBegin(DM, Vec g, InsertMode, Vec l) {
  l->a = g->a;
  return 0;
}
PetscErrorCode DMGlobalToLocalEnd(DM, Vec, InsertMode, Vec) { return 0; }
PetscErrorCode DMLocalToGlobalBegin(DM, Vec l, InsertMode, Vec g) {
  g->a = l->a;
  return 0;
}
PetscErrorCode DMLocalToGlobalEnd(DM, Vec, InsertMode, Vec) { return 0; }
PetscErrorCode VecGetArrayRead(Vec v, const PetscScalar** p) {
  *p = v->a.data();
  return 0;
}
PetscErrorCode VecRestoreArrayRead(Vec, const PetscScalar**) { return 0; }
PetscErrorCode VecGetArray(Vec v, PetscScalar** p) {
  *p = v->a.data();
  return 0;
}
PetscErrorCode VecRestoreArray(Vec, PetscScalar**) { return 0; }
PetscErrorCode VecDestroy(Vec* v) {
  delete *v;
  *v = nullptr;
  return 0;
}
PetscErrorCode VecNormBegin(Vec v, NormType type, PetscReal* norm) {
  double acc = 0.0;
  for (size_t i = 0; i < v->a.size(); ++i) acc += type == NORM_1 ? std::fabs(v->a[i]) : v->a[i] * v->a[i];
  *norm = type == NORM_1 ? acc : std::sqrt(acc);
  return 0;
}
PetscErrorCode VecNormEnd(Vec, NormType, PetscReal*) { return 0; }
int PetscIsInfOrNanReal(PetscReal v) { return std::isnan(v) || std::isinf(v); }
// The harness owns its DM; the limiter's destructor only lets go of it.
PetscErrorCode DMDestroy(DM* dm) {
  *dm = nullptr;
  return 0;
}

// ------------------------------------------------------------- geometry ----
template <typename REAL>
wxNodalDGgeometry2D<REAL>::wxNodalDGgeometry2D(DM dm, unsigned meqn, unsigned Spor)
    : _meqn(meqn), _polyOr(Spor), _dm(dm) {
  _NpE = dm->Np;
  _NpF = dm->N + 1;
  _NfE = 3;
  _totNFace = 0;
  _r = _s = _Ds = _Dr = _Vand = _VVT = nullptr;
  _IVand = nullptr;
  _EtoV = nullptr;
  _Ktotal = _Klocal = _kLocalInt = dm->K;
  _Vlocal = 0;
  _dtscale = _rmin = 0;
  _Mass = new REAL[(size_t)_NpE * _NpE];
  for (int i = 0; i < _NpE * _NpE; ++i) _Mass[i] = (REAL)dm->mass[i];
  _Fmask = new int[_NfE * _NpF];
  for (int i = 0; i < _NfE * _NpF; ++i) _Fmask[i] = dm->fmask[i];
  _xcoord = new REAL*[_Klocal];
  _ycoord = new REAL*[_Klocal];
  _ETETF = new int*[_Klocal];
  for (int k = 0; k < _Klocal; ++k) {
    _xcoord[k] = new REAL[_NpE];
    _ycoord[k] = new REAL[_NpE];
    for (int n = 0; n < _NpE; ++n) {
      _xcoord[k][n] = (REAL)dm->x[(size_t)k * _NpE + n];
      _ycoord[k][n] = (REAL)dm->y[(size_t)k * _NpE + n];
    }
    _ETETF[k] = new int[6];
    for (int f = 0; f < 6; ++f) _ETETF[k][f] = dm->conn[(size_t)k * 6 + f];
  }
}

template <typename REAL>
wxNodalDGgeometry2D<REAL>::~wxNodalDGgeometry2D() {
  for (int k = 0; k < _Klocal; ++k) {
    delete[] _xcoord[k];
    delete[] _ycoord[k];
    delete[] _ETETF[k];
  }
  delete[] _xcoord;
  delete[] _ycoord;
  delete[] _ETETF;
  delete[] _Fmask;
  delete[] _Mass;
}

// wxnodaldggeometry2d.cc:384-410: unit outward normals from the element's
// vertex nodes, and half the edge length, per face
template <typename REAL>
void wxNodalDGgeometry2D<REAL>::Normals2d(int k, REAL norms[]) {
  REAL x1 = _xcoord[k][_Fmask[0 * _NpF]], y1 = _ycoord[k][_Fmask[0 * _NpF]];
  REAL x2 = _xcoord[k][_Fmask[1 * _NpF]], y2 = _ycoord[k][_Fmask[1 * _NpF]];
  REAL x3 = _xcoord[k][_Fmask[2 * _NpF]], y3 = _ycoord[k][_Fmask[2 * _NpF]];
  norms[0] = (y2 - y1);
  norms[1] = -(x2 - x1);
  norms[3] = (y3 - y2);
  norms[4] = -(x3 - x2);
  norms[6] = (y1 - y3);
  norms[7] = -(x1 - x3);
  for (int f = 0; f < _NfE; ++f) {
    REAL sJ = sqrt(norms[_NfE * f] * norms[_NfE * f] + norms[_NfE * f + 1] * norms[_NfE * f + 1]);
    norms[_NfE * f] /= sJ;
    norms[_NfE * f + 1] /= sJ;
    norms[_NfE * f + 2] = sJ / 2.;
  }
}

// wxnodaldggeometry2d.cc:414-438: [dr/dx, ds/dx, dr/dy, ds/dy, J] of the
// affine map from the reference triangle
template <typename REAL>
void wxNodalDGgeometry2D<REAL>::GeometricFactors2d(int k, REAL geom[]) {
  REAL x1 = _xcoord[k][_Fmask[0 * _NpF]], y1 = _ycoord[k][_Fmask[0 * _NpF]];
  REAL x2 = _xcoord[k][_Fmask[1 * _NpF]], y2 = _ycoord[k][_Fmask[1 * _NpF]];
  REAL x3 = _xcoord[k][_Fmask[2 * _NpF]], y3 = _ycoord[k][_Fmask[2 * _NpF]];
  REAL dxdr = (x2 - x1) / 2, dxds = (x3 - x1) / 2;
  REAL dydr = (y2 - y1) / 2, dyds = (y3 - y1) / 2;
  REAL J = -dxds * dydr + dxdr * dyds;
  geom[0] = dyds / J;
  geom[1] = -dydr / J;
  geom[2] = -dxds / J;
  geom[3] = dxdr / J;
  geom[4] = J;
}

template class wxNodalDGgeometry2D<float>;
template class wxNodalDGgeometry2D<double>;

// -------------------------------------------------------------- harness ----
namespace {
std::string g_err;

struct Harness {
  _p_DM dm;
  ApSolver<double>* solver = nullptr;
  wxNodalDGgeometry2D<double>* geom = nullptr;
  WxNodalDGLimiter<double>* limiter = nullptr;
  ~Harness() {
    delete limiter;
    delete geom;
    delete solver;  // deletes the boundary conditions it holds
  }
};

}  // namespace

extern "C" {
const char* reflim_last_error() { return g_err.c_str(); }

// A mesh of K elements at order N with meqn fields per node: node coordinates
// x, y [K][Np], the element-to-element-to-face table conn [K][6] in Apollo's
// _ETETF convention (neighbour and its face, or -tag twice on a boundary
// face), the face masks fmask [3 (N+1)] and the reference element's mass
// matrix [Np][Np].
void* reflim_create(int K, int N, int meqn, const double* x, const double* y, const int* conn, const int* fmask,
                    const double* mass) {
  Harness* h = new Harness();
  const int Np = (N + 1) * (N + 2) / 2;
  h->dm.K = K;
  h->dm.N = N;
  h->dm.Np = Np;
  h->dm.dof = Np * meqn;
  h->dm.x.assign(x, x + (size_t)K * Np);
  h->dm.y.assign(y, y + (size_t)K * Np);
  h->dm.conn.assign(conn, conn + (size_t)K * 6);
  h->dm.fmask.assign(fmask, fmask + 3 * (N + 1));
  h->dm.mass.assign(mass, mass + (size_t)Np * Np);
  h->solver = new ApSolver<double>("harness");
  h->geom = new wxNodalDGgeometry2D<double>(&h->dm, (unsigned)meqn, (unsigned)N);
  return h;
}

void reflim_destroy(void* p) { delete (Harness*)p; }

// One boundary-condition plugin of the registered kind, set up from a
// cryptset holding its keys under one top-level set whose name names it.
int reflim_add_bc(void* p, const char* kind, const char* text) {
  Harness* h = (Harness*)p;
  ApSubSolver<double>* bc = make_bc(kind);
  if (!bc) {
    g_err = std::string("unknown boundary condition kind ") + kind;
    return -1;
  }
  try {
    std::istringstream in(text);
    WxCryptSet wxc(in);
    bc->setup(wxc, &h->dm);
    bc->setParent(h->solver);
    g_pending.push_back(std::make_pair(wxc.name(), bc));
    h->solver->init();
  } catch (...) {
    delete bc;
    g_err = "boundary condition setup failed";
    return -1;
  }
  return 0;
}

// The boundary condition registered under `name` at one point:
// WxGridBC::applyToArray(xc, nx, q, 0, 0, qBC) (wxgridbc.cc).
int reflim_apply_bc(void* p, const char* name, const double* xc, const double* nx, const double* q, int meqn,
                    double* qbc) {
  Harness* h = (Harness*)p;
  try {
    WxGridBC<double>* bc = dynamic_cast<WxGridBC<double>*>(h->solver->getSubSolver(name));
    if (!bc) return -1;
    double xx[5] = {xc[0], xc[1], xc[2], xc[3], xc[4]}, nn[3] = {nx[0], nx[1], 0.0}, qq[16];
    std::memcpy(qq, q, meqn * sizeof(double));
    bc->applyToArray(xx, nn, qq, nullptr, nullptr, qbc);
  } catch (...) {
    g_err = std::string("no boundary condition ") + name;
    return -1;
  }
  return 0;
}

// A limiter set up from its cryptset block: kind 0 eulerLimiterHW
// (gas_gamma, min_pressure, min_density, boundaryConditions naming registered
// conditions in tag order), kind 1 tuAliabadiLimiter (boundaryConditions and
// the `Equations` list with the equations' own sets).
int reflim_set_limiter(void* p, int kind, const char* text) {
  Harness* h = (Harness*)p;
  try {
    std::istringstream in(text);
    WxCryptSet wxc(in);
    WxNodalDGLimiter<double>* lim;
    if (kind == 0) lim = new WxHestavenWarburtonEulerLimiter<double>();
    else lim = new WxTuAliabadiLimiter<double>();
    ApSubSolver<double>* base = lim;
    base->setup(wxc, &h->dm);
    lim->setParent(h->solver);
    delete h->limiter;
    h->limiter = lim;
  } catch (...) {
    g_err = "limiter setup failed";
    return -1;
  }
  return 0;
}

// Apollo's limiter on u [K][Np][meqn] into out (WxNodalDGLimiter::applyToVector).
int reflim_limit(void* p, const double* u, double* out) {
  Harness* h = (Harness*)p;
  if (!h->limiter) return -1;
  const size_t n = (size_t)h->dm.K * h->dm.dof;
  _p_Vec in, res;
  in.a.assign(u, u + n);
  res.a.assign(n, 0.0);
  try {
    h->limiter->applyToVector(h->geom, nullptr, &in, &res);
  } catch (...) {
    g_err = "limiter failed";
    return -1;
  }
  std::memcpy(out, res.a.data(), n * sizeof(double));
  return 0;
}
}  // extern "C"
