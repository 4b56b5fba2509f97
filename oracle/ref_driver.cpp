// ORACLE — test infrastructure only.  Runs Apollo's own nodal-DG right-hand
// side, compiled unmodified from the Apollo source tree by `oracle/Makefile
// refdrv` into oracle/_ref/libapollo_refdrv.so, so that tests can check the
// oracle's restatement of the whole right-hand-side path against Apollo's
// code:
//   WxNodalDG2dMethod::setup/init/step   src/subsolvers/wxnodaldg2dmethod.cc:53-542
//   wxNodalDGgeometry2D                  src/lib/wxnodaldggeometry2d.cc (nodes,
//                                        matrices, connectivity, normals, factors)
//   WxCubature2d                         src/lib/wxcubature2d.cc (cubature and
//                                        Gauss interpolation, volume and surface
//                                        integrals)
//   wxpnodaldgfunctions.h, wxNodalDGMatrices.h (node sets, Vandermonde and
//   derivative matrices), the equation, source and area-integral sets, the
//   grid boundary conditions and the limiters with their bases (a limiter
//   named in the method's `Limiter` list acts on the step's input, as
//   WxNodalDG2dMethod::step does).
//
// What this file supplies in place of PETSc and MPI (declared in
// solver_stub/petsc.h and solver_stub/mpi.h):
//   * dense matrices with PETSc's calling conventions (and sparse ones for the
//     face-to-vertex and face-to-face connectivity): products summed in
//     index order, LU with partial pivoting and the triangular solves in the
//     order of LAPACK's unblocked dgetf2/dgetrs (PETSc's dense LU calls
//     LAPACK; which LAPACK Apollo links is not known, so results agree with
//     the oracle to round-off, not bit for bit);
//   * a DMPlex-shaped mesh: cells [0, K), vertices [K, K + V), edges after
//     them, each cell's cone its three vertices in the caller's order, a
//     "Face Sets" label on boundary edges, one section of Np x meqn values
//     per cell, and no ghost cells (DMPlexGetHybridBounds returns K);
//   * vectors over that section, and MPI for one process.
#include <cmath>
#include <cstring>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include <wxcreator.h>
#include <wxcryptset.h>
#include <wxexprfunction.h>
#include <wxnodaldg2dmethod.h>
#include "advection/wxadvectioneqn.h"
#include "euler/wxeulereqn.h"
#include "maxwell/wxphmaxwelleqn.h"
#include "maxwell/wxpointcurrent.h"
#include "maxwell/wxtransversemagneticsrc.h"
#include "euler/wxhesthavenwarburtoneulerlimiter.h"
#include "multifluid/aptualiabadilimiter.h"
#include "ref_harness.h"

// The plugin kinds under their Apollo names (aphyperapps_register.cc,
// wxfunction_register.cc).
static WxCreator<WxAdvectionEqn<double>, WxHyperbolicEqn<double> > reg_adv("advectionEqn");
static WxCreator<WxEulerEqn<double>, WxHyperbolicEqn<double> > reg_euler("eulerEqn");
static WxCreator<WxPHMaxwellEqn<double>, WxHyperbolicEqn<double> > reg_maxwell("phMaxwellEqn");
static WxCreator<WxTransverseMagneticSrc<double>, WxHyperbolicSrc<double> > reg_tmsrc("tranverseMagneticSrc");
static WxCreator<WxpointCurrentSrc<double>, WxHyperbolicSrc<double> > reg_pcsrc("pointCurrentSrc");
static WxCreator<WxExprFunc, WxFunction<double> > reg_expr("exprFunc");

// ------------------------------------------------------------------- MPI ----
static size_t mpi_size(MPI_Datatype t) {
  switch (t) {
    case MPI_INT: case MPI_UNSIGNED: case MPI_FLOAT: return 4;
    case MPI_DOUBLE: case MPI_LONG: case MPI_UNSIGNED_LONG: case MPI_LONG_LONG_INT: return 8;
    case MPI_SHORT: case MPI_UNSIGNED_SHORT: return 2;
    case MPI_LONG_DOUBLE: return sizeof(long double);
    default: return 1;
  }
}
int MPI_Allreduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op, MPI_Comm) {
  std::memmove(r, s, (size_t)n * mpi_size(t));
  return 0;
}
int MPI_Comm_rank(MPI_Comm, int* rank) { *rank = 0; return 0; }
int MPI_Comm_size(MPI_Comm, int* size) { *size = 1; return 0; }
int MPI_Barrier(MPI_Comm) { return 0; }

// ---------------------------------------------------------------- matrix ----
struct _p_Mat {
  int m = 0, n = 0;
  std::vector<double> a;    // row-major
  std::vector<int> cols;    // 0 .. n-1, what MatGetRow hands out
  std::vector<double> lu;   // a factor: LU of the factored matrix, row-major
  std::vector<int> piv;     // and its row interchanges
  // a sparse (AIJ) matrix: its rows, and the row MatGetRow last handed out
  bool aij = false;
  std::vector<std::map<int, double> > sp;
  std::vector<int> rc;
  std::vector<double> rv;
  void shape(int mm, int nn) {
    m = mm; n = nn;
    a.assign((size_t)m * n, 0.0);
    cols.resize(n);
    for (int j = 0; j < n; ++j) cols[j] = j;
  }
};
static Mat new_mat(int m, int n) {
  Mat A = new _p_Mat();
  A->shape(m, n);
  return A;
}
PetscErrorCode MatCreateSeqDense(MPI_Comm, PetscInt m, PetscInt n, PetscScalar*, Mat* A) {
  *A = new_mat(m, n);
  return 0;
}
PetscErrorCode MatCreateSeqAIJ(MPI_Comm, PetscInt m, PetscInt n, PetscInt, const PetscInt*, Mat* A) {
  *A = new _p_Mat();
  (*A)->m = m;
  (*A)->n = n;
  (*A)->aij = true;
  (*A)->sp.resize(m);
  return 0;
}
PetscErrorCode MatSetValue(Mat A, PetscInt i, PetscInt j, PetscScalar v, InsertMode mode) {
  double& x = A->aij ? A->sp[i][j] : A->a[(size_t)i * A->n + j];
  x = mode == ADD_VALUES ? x + v : v;
  return 0;
}
PetscErrorCode MatAssemblyBegin(Mat, MatAssemblyType) { return 0; }
PetscErrorCode MatAssemblyEnd(Mat, MatAssemblyType) { return 0; }
// A dense row: every column, as PETSc's dense MatGetRow gives it; a sparse
// row: its stored entries in column order.
PetscErrorCode MatGetRow(Mat A, PetscInt r, PetscInt* nc, const PetscInt** c, const PetscScalar** v) {
  if (A->aij) {
    A->rc.clear();
    A->rv.clear();
    for (std::map<int, double>::const_iterator it = A->sp[r].begin(); it != A->sp[r].end(); ++it) {
      A->rc.push_back(it->first);
      A->rv.push_back(it->second);
    }
    *nc = (PetscInt)A->rc.size();
    if (c) *c = A->rc.data();
    if (v) *v = A->rv.data();
    return 0;
  }
  *nc = A->n;
  if (c) *c = A->cols.data();
  if (v) *v = &A->a[(size_t)r * A->n];
  return 0;
}
PetscErrorCode MatRestoreRow(Mat, PetscInt, PetscInt*, const PetscInt**, const PetscScalar**) { return 0; }
PetscErrorCode MatGetSize(Mat A, PetscInt* m, PetscInt* n) {
  if (m) *m = A->m;
  if (n) *n = A->n;
  return 0;
}
PetscErrorCode MatDestroy(Mat* A) {
  delete *A;
  *A = nullptr;
  return 0;
}
PetscErrorCode MatView(Mat, PetscViewer) { return 0; }
PetscErrorCode MatZeroEntries(Mat A) {
  std::fill(A->a.begin(), A->a.end(), 0.0);
  for (size_t i = 0; i < A->sp.size(); ++i)
    for (std::map<int, double>::iterator it = A->sp[i].begin(); it != A->sp[i].end(); ++it) it->second = 0.0;
  return 0;
}
PetscErrorCode MatTranspose(Mat A, MatReuse reuse, Mat* B) {
  if (reuse != MAT_REUSE_MATRIX || !*B) *B = new_mat(A->n, A->m);
  for (int i = 0; i < A->m; ++i)
    for (int j = 0; j < A->n; ++j) (*B)->a[(size_t)j * A->m + i] = A->a[(size_t)i * A->n + j];
  return 0;
}
// C = A B (or A B^T), each entry summed over the inner index in order
static void matmul(Mat A, Mat B, bool bt, MatReuse reuse, Mat* C) {
  const int m = A->m, k = A->n, n = bt ? B->m : B->n;
  if (reuse != MAT_REUSE_MATRIX || !*C) *C = new_mat(m, n);
  else if ((*C)->m != m || (*C)->n != n) (*C)->shape(m, n);
  for (int i = 0; i < m; ++i)
    for (int j = 0; j < n; ++j) {
      double s = 0.0;
      for (int l = 0; l < k; ++l) s += A->a[(size_t)i * k + l] * (bt ? B->a[(size_t)j * k + l] : B->a[(size_t)l * n + j]);
      (*C)->a[(size_t)i * n + j] = s;
    }
}
PetscErrorCode MatMatMult(Mat A, Mat B, MatReuse reuse, PetscReal, Mat* C) {
  matmul(A, B, false, reuse, C);
  return 0;
}
// Sparse A B^T (the face-to-face connectivity from face-to-vertex): the
// pattern of every pair of rows sharing a column, as PETSc's AIJ product has it
PetscErrorCode MatMatTransposeMult(Mat A, Mat B, MatReuse reuse, PetscReal, Mat* C) {
  if (!A->aij || !B->aij) {
    matmul(A, B, true, reuse, C);
    return 0;
  }
  std::vector<std::vector<std::pair<int, double> > > bcol(B->n);
  for (int j = 0; j < B->m; ++j)
    for (std::map<int, double>::const_iterator it = B->sp[j].begin(); it != B->sp[j].end(); ++it)
      bcol[it->first].push_back(std::make_pair(j, it->second));
  MatCreateSeqAIJ(MPI_COMM_SELF, A->m, B->m, 0, nullptr, C);
  for (int i = 0; i < A->m; ++i)
    for (std::map<int, double>::const_iterator it = A->sp[i].begin(); it != A->sp[i].end(); ++it)
      for (size_t q = 0; q < bcol[it->first].size(); ++q)
        (*C)->sp[i][bcol[it->first][q].first] += it->second * bcol[it->first][q].second;
  return 0;
}
PetscErrorCode MatDuplicate(Mat A, MatDuplicateOption op, Mat* B) {
  *B = new_mat(A->m, A->n);
  if (op == MAT_COPY_VALUES) (*B)->a = A->a;
  return 0;
}
PetscErrorCode MatGetFactor(Mat A, const char*, MatFactorType, Mat* F) {
  *F = new_mat(A->m, A->n);
  return 0;
}
PetscErrorCode MatLUFactorSymbolic(Mat, Mat, IS, IS, const MatFactorInfo*) { return 0; }
// LU with partial pivoting (the first largest magnitude), the column below
// the pivot scaled by its reciprocal, then the rank-one update: dgetf2's order
PetscErrorCode MatLUFactorNumeric(Mat F, Mat A, const MatFactorInfo*) {
  const int n = A->n;
  F->lu = A->a;
  F->piv.assign(n, 0);
  double* a = F->lu.data();
  for (int j = 0; j < n; ++j) {
    int p = j;
    double best = std::fabs(a[(size_t)j * n + j]);
    for (int i = j + 1; i < n; ++i)
      if (std::fabs(a[(size_t)i * n + j]) > best) { best = std::fabs(a[(size_t)i * n + j]); p = i; }
    F->piv[j] = p;
    if (p != j)
      for (int c = 0; c < n; ++c) std::swap(a[(size_t)j * n + c], a[(size_t)p * n + c]);
    const double r = 1.0 / a[(size_t)j * n + j];
    for (int i = j + 1; i < n; ++i) a[(size_t)i * n + j] *= r;
    for (int i = j + 1; i < n; ++i)
      for (int c = j + 1; c < n; ++c) a[(size_t)i * n + c] -= a[(size_t)i * n + j] * a[(size_t)j * n + c];
  }
  return 0;
}
PetscErrorCode MatLUFactor(Mat A, IS, IS, const MatFactorInfo*) { return MatLUFactorNumeric(A, A, nullptr); }
// X = A^-1 B from the factor: row interchanges, unit lower solve, upper solve
// from the last row up (dgetrs)
PetscErrorCode MatMatSolve(Mat F, Mat B, Mat X) {
  const int n = F->n, nr = B->n;
  std::vector<double> x = B->a;
  for (int j = 0; j < n; ++j)
    if (F->piv[j] != j)
      for (int c = 0; c < nr; ++c) std::swap(x[(size_t)j * nr + c], x[(size_t)F->piv[j] * nr + c]);
  const double* a = F->lu.data();
  for (int c = 0; c < nr; ++c) {
    for (int k = 0; k < n; ++k) {
      const double xk = x[(size_t)k * nr + c];
      if (xk != 0.0)
        for (int i = k + 1; i < n; ++i) x[(size_t)i * nr + c] -= xk * a[(size_t)i * n + k];
    }
    for (int k = n - 1; k >= 0; --k) {
      if (x[(size_t)k * nr + c] != 0.0) {
        x[(size_t)k * nr + c] /= a[(size_t)k * n + k];
        const double xk = x[(size_t)k * nr + c];
        for (int i = 0; i < k; ++i) x[(size_t)i * nr + c] -= xk * a[(size_t)i * n + k];
      }
    }
  }
  if (X->m != n || X->n != nr) X->shape(n, nr);
  X->a = x;
  return 0;
}

// ------------------------------------------------------------------ mesh ----
struct _p_PetscSection {
  int dof = 0;  // values per cell
};
struct _p_Vec {
  std::vector<double> a;
  DM dm = nullptr;
};
struct _p_DM {
  int K = 0, V = 0, E = 0, dof = 0;
  bool uninterpolated = false;
  _p_DM* unint = nullptr;           // the uninterpolated view (shares the data)
  std::vector<int> cone;            // [K][3] vertex points
  std::vector<int> support;         // [E][2] cells (-1 for none)
  std::vector<int> label;           // [E] "Face Sets" value, -1 for none
  _p_Vec coords;                    // [V][2]
  _p_PetscSection section, csection;
};

PetscErrorCode DMPlexGetHeightStratum(DM dm, PetscInt h, PetscInt* s, PetscInt* e) {
  if (h == 0) { *s = 0; *e = dm->K; }
  else { *s = dm->K + dm->V; *e = dm->K + dm->V + dm->E; }
  return 0;
}
PetscErrorCode DMPlexGetDepthStratum(DM dm, PetscInt d, PetscInt* s, PetscInt* e) {
  if (d == 0) { *s = dm->K; *e = dm->K + dm->V; }
  else if (d == 1) { *s = dm->K + dm->V; *e = dm->K + dm->V + dm->E; }
  else { *s = 0; *e = dm->K; }
  return 0;
}
PetscErrorCode DMPlexGetHybridBounds(DM dm, PetscInt* c, PetscInt* f, PetscInt* e, PetscInt* v) {
  if (c) *c = dm->K;
  if (f) *f = -1;
  if (e) *e = -1;
  if (v) *v = -1;
  return 0;
}
PetscErrorCode DMPlexUninterpolate(DM dm, DM* u) {
  *u = dm->unint;
  return 0;
}
PetscErrorCode DMPlexGetCone(DM dm, PetscInt p, const PetscInt** cone) {
  *cone = &dm->cone[(size_t)p * 3];
  return 0;
}
PetscErrorCode DMPlexGetSupport(DM dm, PetscInt p, const PetscInt** cells) {
  *cells = &dm->support[(size_t)(p - dm->K - dm->V) * 2];
  return 0;
}
PetscErrorCode DMPlexGetLabelValue(DM dm, const char* name, PetscInt p, PetscInt* v) {
  const int e = p - dm->K - dm->V;
  *v = (std::string(name) == "Face Sets" && e >= 0 && e < dm->E) ? dm->label[e] : -1;
  return 0;
}
PetscErrorCode DMGetCoordinatesLocal(DM dm, Vec* v) {
  *v = &dm->coords;
  return 0;
}
PetscErrorCode DMGetCoordinateSection(DM dm, PetscSection* s) {
  *s = &dm->csection;
  return 0;
}
PetscErrorCode DMGetDefaultSection(DM dm, PetscSection* s) {
  *s = &dm->section;
  return 0;
}
PetscErrorCode PetscSectionGetOffset(PetscSection s, PetscInt p, PetscInt* off) {
  *off = p * s->dof;
  return 0;
}
PetscErrorCode DMPlexVecGetClosure(DM, PetscSection, Vec, PetscInt, PetscInt*, PetscScalar**) { return 1; }
PetscErrorCode DMPlexVecRestoreClosure(DM, PetscSection, Vec, PetscInt, PetscInt*, PetscScalar**) { return 0; }
PetscErrorCode DMPlexPointLocalRead(DM dm, PetscInt p, const PetscScalar* a, void* ptr) {
  *(const PetscScalar**)ptr = a + (size_t)p * dm->dof;
  return 0;
}
PetscErrorCode DMPlexPointLocalRef(DM dm, PetscInt p, PetscScalar* a, void* ptr) {
  *(PetscScalar**)ptr = a + (size_t)p * dm->dof;
  return 0;
}
PetscErrorCode DMPlexPointGlobalRef(DM dm, PetscInt p, PetscScalar* a, void* ptr) {
  *(PetscScalar**)ptr = a + (size_t)p * dm->dof;
  return 0;
}
PetscErrorCode DMGetLocalVector(DM dm, Vec* v) {
  *v = new _p_Vec();
  (*v)->a.assign((size_t)dm->K * dm->dof, 0.0);
  (*v)->dm = dm;
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
// The harness owns its meshes; Apollo's destroy calls only let go of them.
PetscErrorCode DMDestroy(DM* dm) {
  *dm = nullptr;
  return 0;
}

// --------------------------------------------------------------- vectors ----
PetscErrorCode VecGetArrayRead(Vec v, const PetscScalar** p) { *p = v->a.data(); return 0; }
PetscErrorCode VecRestoreArrayRead(Vec, const PetscScalar**) { return 0; }
PetscErrorCode VecGetArray(Vec v, PetscScalar** p) { *p = v->a.data(); return 0; }
PetscErrorCode VecRestoreArray(Vec, PetscScalar**) { return 0; }
PetscErrorCode VecDestroy(Vec* v) {
  delete *v;
  *v = nullptr;
  return 0;
}
PetscErrorCode VecCreateSeq(MPI_Comm, PetscInt n, Vec* v) {
  *v = new _p_Vec();
  (*v)->a.assign(n, 0.0);
  return 0;
}
PetscErrorCode VecGetSize(Vec v, PetscInt* n) { *n = (PetscInt)v->a.size(); return 0; }
PetscErrorCode VecZeroEntries(Vec v) {
  std::fill(v->a.begin(), v->a.end(), 0.0);
  return 0;
}
PetscErrorCode VecDuplicate(Vec v, Vec* w) {
  *w = new _p_Vec();
  (*w)->a.assign(v->a.size(), 0.0);
  (*w)->dm = v->dm;
  return 0;
}
PetscErrorCode VecGetDM(Vec v, DM* dm) { *dm = v->dm; return 0; }
PetscErrorCode VecView(Vec, PetscViewer) { return 0; }
PetscErrorCode VecNormBegin(Vec v, NormType type, PetscReal* norm) {
  double acc = 0.0;
  for (size_t i = 0; i < v->a.size(); ++i) acc += type == NORM_1 ? std::fabs(v->a[i]) : v->a[i] * v->a[i];
  *norm = type == NORM_1 ? acc : std::sqrt(acc);
  return 0;
}
PetscErrorCode VecNormEnd(Vec, NormType, PetscReal*) { return 0; }
int PetscIsInfOrNanReal(PetscReal v) { return std::isnan(v) || std::isinf(v); }
MPI_Comm PetscObjectComm(PetscObject) { return MPI_COMM_WORLD; }
PetscErrorCode PetscBarrier(PetscObject) { return 0; }
PetscErrorCode PetscFinalize(void) { return 0; }

// --------------------------------------------------------------- harness ----
namespace {
std::string g_err;

struct Driver {
  _p_DM dm, unint;
  ApSolver<double>* solver = nullptr;
  WxNodalDG2dMethod<double>* method = nullptr;
  int Np = 0, meqn = 0;
  ~Driver() {
    delete method;
    delete solver;
  }
};
}  // namespace

extern "C" {
const char* refdrv_last_error() { return g_err.c_str(); }

// A triangle mesh: vertices (vx, vy), elements etov [K][3] (counter-clockwise),
// boundary tags face_tag [K][3] (face f joins vertices f and f + 1; 0 for an
// interior face, else the 1-based boundary condition).
void* refdrv_create(int nverts, const double* vx, const double* vy, int K, const int* etov, const int* face_tag) {
  Driver* d = new Driver();
  _p_DM& dm = d->dm;
  dm.K = K;
  dm.V = nverts;
  dm.cone.resize((size_t)K * 3);
  for (int i = 0; i < K * 3; ++i) dm.cone[i] = K + etov[i];
  dm.coords.a.resize((size_t)nverts * 2);
  for (int v = 0; v < nverts; ++v) {
    dm.coords.a[2 * v] = vx[v];
    dm.coords.a[2 * v + 1] = vy[v];
  }
  std::map<std::pair<int, int>, int> edges;
  for (int k = 0; k < K; ++k)
    for (int f = 0; f < 3; ++f) {
      int a = etov[k * 3 + f], b = etov[k * 3 + (f + 1) % 3];
      std::pair<int, int> key(a < b ? a : b, a < b ? b : a);
      std::map<std::pair<int, int>, int>::iterator it = edges.find(key);
      if (it == edges.end()) {
        edges[key] = dm.E++;
        dm.support.push_back(k);
        dm.support.push_back(-1);
        dm.label.push_back(face_tag[k * 3 + f] > 0 ? face_tag[k * 3 + f] : -1);
      } else {
        dm.support[(size_t)it->second * 2 + 1] = k;
      }
    }
  d->unint = dm;
  d->unint.uninterpolated = true;
  dm.unint = &d->unint;
  d->unint.unint = &d->unint;
  d->solver = new ApSolver<double>("harness");
  return d;
}

void refdrv_destroy(void* p) { delete (Driver*)p; }

// One boundary-condition plugin of the registered kind, set up from a
// cryptset holding its keys under one top-level set whose name names it.
int refdrv_add_bc(void* p, const char* kind, const char* text) {
  Driver* d = (Driver*)p;
  ApSubSolver<double>* bc = make_bc(kind);
  if (!bc) {
    g_err = std::string("unknown boundary condition kind ") + kind;
    return -1;
  }
  try {
    std::istringstream in(text);
    WxCryptSet wxc(in);
    bc->setup(wxc, &d->dm);
    bc->setParent(d->solver);
    g_pending.push_back(std::make_pair(wxc.name(), bc));
    d->solver->init();
  } catch (...) {
    delete bc;
    g_err = "boundary condition setup failed";
    return -1;
  }
  return 0;
}

// A limiter sub-solver (kind 0 eulerLimiterHW, 1 tuAliabadiLimiter) set up
// from its cryptset block and registered under the block's name, for the
// method's `Limiter` list.
int refdrv_add_limiter(void* p, int kind, const char* text) {
  Driver* d = (Driver*)p;
  WxNodalDGLimiter<double>* lim = nullptr;
  try {
    std::istringstream in(text);
    WxCryptSet wxc(in);
    if (kind == 0) lim = new WxHestavenWarburtonEulerLimiter<double>();
    else lim = new WxTuAliabadiLimiter<double>();
    ApSubSolver<double>* base = lim;
    base->setup(wxc, &d->dm);
    lim->setParent(d->solver);
    g_pending.push_back(std::make_pair(wxc.name(), base));
    d->solver->init();
  } catch (...) {
    delete lim;
    g_err = "limiter setup failed";
    return -1;
  }
  return 0;
}

// WxNodalDG2dMethod::setup from the sub-solver's cryptset block
// (polynomialOrder, cfl, Equations and their sets, DataStructure,
// InitialCondition, boundaryConditions, optional Sources).
int refdrv_setup(void* p, const char* text) {
  Driver* d = (Driver*)p;
  try {
    std::istringstream in(text);
    WxCryptSet wxc(in);
    WxNodalDG2dMethod<double>* m = new WxNodalDG2dMethod<double>();
    m->setParent(d->solver);
    d->dm.dof = 0;  // set below, once the equations are known
    const int N = wxc.template get<int>("polynomialOrder");
    d->Np = (N + 1) * (N + 2) / 2;
    m->setup(wxc, &d->dm);
    d->meqn = (int)m->totalEqns();
    d->dm.dof = d->Np * d->meqn;
    d->unint.dof = d->dm.dof;
    d->dm.section.dof = d->dm.dof;
    delete d->method;
    d->method = m;
  } catch (WxExcept&) {
    // (WxExcept::what() hands out a pointer into a temporary string,
    // wxexcept.cc:46-49, so its text is not read here)
    g_err = "setup failed: Apollo raised WxExcept (a missing or malformed key, or an unknown Kind)";
    return -1;
  } catch (...) {
    g_err = "setup failed";
    return -1;
  }
  return 0;
}

int refdrv_np(void* p) { return ((Driver*)p)->Np; }
int refdrv_meqn(void* p) { return ((Driver*)p)->meqn; }

// WxNodalDG2dMethod::init at time t: the initial state [K][Np][meqn] and the
// initial dt it sets.
int refdrv_init(void* p, double t, double* u0, double* dt0) {
  Driver* d = (Driver*)p;
  _p_Vec out;
  out.a.assign((size_t)d->dm.K * d->dm.dof, 0.0);
  out.dm = &d->dm;
  try {
    d->method->setCurrentTime(t);
    d->method->init(0.0, &out);
  } catch (...) {
    g_err = "init failed";
    return -1;
  }
  std::memcpy(u0, out.a.data(), out.a.size() * sizeof(double));
  *dt0 = d->method->getDt();
  return 0;
}

// WxNodalDG2dMethod::step(t, dt, u, rhs): the right-hand side and the
// suggested dt.  With a limiter the method limits its input vector in place,
// as it does PETSc's stage vector; that limited input is written back to u.
int refdrv_rhs(void* p, double t, double dt, double* u, double* rhs, double* sugg) {
  Driver* d = (Driver*)p;
  _p_Vec in, out;
  in.a.assign(u, u + (size_t)d->dm.K * d->dm.dof);
  in.dm = &d->dm;
  out.a.assign(in.a.size(), 0.0);
  out.dm = &d->dm;
  try {
    WxStepperStatus<double> st = d->method->step(t, dt, &in, &out);
    *sugg = st.getSuggestedDt();
  } catch (...) {
    g_err = "step failed";
    return -1;
  }
  std::memcpy(rhs, out.a.data(), out.a.size() * sizeof(double));
  std::memcpy(u, in.a.data(), in.a.size() * sizeof(double));
  return 0;
}
}  // extern "C"
