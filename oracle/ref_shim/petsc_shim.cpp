// Single-rank implementation of the DMDA subset declared in petscdmda.h.
// Test infrastructure for compiling the reference M2C sources as a CPU oracle.
#include <petscdmda.h>

#include <cstdarg>
#include <cstdlib>
#include <cstring>
#include <vector>

MPI_Comm PETSC_COMM_WORLD = 0;

struct m2c_shim_dm {
  int NX, NY, NZ, dof, s;
  DMBoundaryType bx, by, bz;
};

struct m2c_shim_vec {
  DM dm;
  bool local;              // ghosted box (local) or interior only (global)
  int gx0, gy0, gz0;       // lowest index held (−s for local, 0 for global)
  int gnx, gny, gnz;       // extent held
  std::vector<double> data;
  std::vector<double*> rows;    // [gnz*gny] row pointers offset by −gx0*dof
  std::vector<double**> planes; // [gnz] plane pointers offset by −gy0
};

PetscErrorCode PetscInitialize(int*, char***, const char*, const char*) { return 0; }
PetscErrorCode PetscFinalize() { return 0; }
PetscErrorCode PetscPrintf(MPI_Comm, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vfprintf(stdout, fmt, ap);
  va_end(ap);
  return 0;
}

PetscErrorCode DMDACreate3d(MPI_Comm, DMBoundaryType bx, DMBoundaryType by, DMBoundaryType bz,
                            DMDAStencilType, PetscInt M, PetscInt N, PetscInt P, PetscInt, PetscInt,
                            PetscInt, PetscInt dof, PetscInt s, const PetscInt*, const PetscInt*,
                            const PetscInt*, DM* da) {
  DM d = new m2c_shim_dm;
  d->NX = M; d->NY = N; d->NZ = P; d->dof = dof; d->s = s;
  d->bx = bx; d->by = by; d->bz = bz;
  *da = d;
  return 0;
}
PetscErrorCode DMSetFromOptions(DM) { return 0; }
PetscErrorCode DMSetUp(DM) { return 0; }
PetscErrorCode DMDestroy(DM* d) { delete *d; *d = nullptr; return 0; }

PetscErrorCode DMDAGetInfo(DM d, PetscInt* dim, PetscInt* M, PetscInt* N, PetscInt* P, PetscInt* m,
                           PetscInt* n, PetscInt* p, PetscInt* dof, PetscInt* s, DMBoundaryType* bx,
                           DMBoundaryType* by, DMBoundaryType* bz, DMDAStencilType* st) {
  if (dim) *dim = 3;
  if (M) *M = d->NX;
  if (N) *N = d->NY;
  if (P) *P = d->NZ;
  if (m) *m = 1;
  if (n) *n = 1;
  if (p) *p = 1;
  if (dof) *dof = d->dof;
  if (s) *s = d->s;
  if (bx) *bx = d->bx;
  if (by) *by = d->by;
  if (bz) *bz = d->bz;
  if (st) *st = DMDA_STENCIL_BOX;
  return 0;
}

PetscErrorCode DMDAGetCorners(DM d, PetscInt* x, PetscInt* y, PetscInt* z, PetscInt* m, PetscInt* n,
                              PetscInt* p) {
  if (x) *x = 0;
  if (y) *y = 0;
  if (z) *z = 0;
  if (m) *m = d->NX;
  if (n) *n = d->NY;
  if (p) *p = d->NZ;
  return 0;
}

static int ghost_of(DMBoundaryType b, int s) { return b == DM_BOUNDARY_NONE ? 0 : s; }

PetscErrorCode DMDAGetGhostCorners(DM d, PetscInt* x, PetscInt* y, PetscInt* z, PetscInt* m,
                                   PetscInt* n, PetscInt* p) {
  int sx = ghost_of(d->bx, d->s), sy = ghost_of(d->by, d->s), sz = ghost_of(d->bz, d->s);
  if (x) *x = -sx;
  if (y) *y = -sy;
  if (z) *z = -sz;
  if (m) *m = d->NX + 2 * sx;
  if (n) *n = d->NY + 2 * sy;
  if (p) *p = d->NZ + 2 * sz;
  return 0;
}

static Vec make_vec(DM d, bool local) {
  Vec v = new m2c_shim_vec;
  v->dm = d;
  v->local = local;
  if (local) {
    DMDAGetGhostCorners(d, &v->gx0, &v->gy0, &v->gz0, &v->gnx, &v->gny, &v->gnz);
  } else {
    v->gx0 = v->gy0 = v->gz0 = 0;
    v->gnx = d->NX; v->gny = d->NY; v->gnz = d->NZ;
  }
  size_t row = (size_t)v->gnx * d->dof;
  v->data.assign(row * v->gny * v->gnz, 0.0);
  v->rows.resize((size_t)v->gny * v->gnz);
  v->planes.resize(v->gnz);
  for (int k = 0; k < v->gnz; k++) {
    for (int j = 0; j < v->gny; j++)
      v->rows[(size_t)k * v->gny + j] = v->data.data() + ((size_t)k * v->gny + j) * row - (long)v->gx0 * d->dof;
    v->planes[k] = v->rows.data() + (size_t)k * v->gny - v->gy0;
  }
  return v;
}

PetscErrorCode DMCreateGlobalVector(DM d, Vec* v) { *v = make_vec(d, false); return 0; }
PetscErrorCode DMCreateLocalVector(DM d, Vec* v) { *v = make_vec(d, true); return 0; }
PetscErrorCode VecSet(Vec v, PetscScalar a) {
  for (auto& x : v->data) x = a;
  return 0;
}
PetscErrorCode VecDestroy(Vec* v) { delete *v; *v = nullptr; return 0; }

PetscErrorCode DMDAVecGetArray(DM, Vec v, void* array) {
  *(double****)array = v->planes.data() - v->gz0;
  return 0;
}
PetscErrorCode DMDAVecRestoreArray(DM, Vec, void* array) {
  *(double****)array = nullptr;
  return 0;
}

// Interior of the local vector <-> global vector.
static void interior_transfer(DM d, Vec l, Vec g, bool to_global, bool add) {
  size_t row = (size_t)d->NX * d->dof;
  for (int k = 0; k < d->NZ; k++)
    for (int j = 0; j < d->NY; j++) {
      double* lp = l->planes[k - l->gz0][j];
      double* gp = g->planes[k][j];
      if (to_global) {
        if (add)
          for (size_t q = 0; q < row; q++) gp[q] += lp[q];
        else
          memcpy(gp, lp, row * sizeof(double));
      } else {
        memcpy(lp, gp, row * sizeof(double));
      }
    }
}

PetscErrorCode DMLocalToGlobal(DM d, Vec l, InsertMode mode, Vec g) {
  interior_transfer(d, l, g, true, mode == ADD_VALUES);
  return 0;
}
PetscErrorCode DMGlobalToLocalBegin(DM, Vec, InsertMode, Vec) { return 0; }
PetscErrorCode DMGlobalToLocalEnd(DM d, Vec g, InsertMode, Vec l) {
  interior_transfer(d, l, g, false, false);
  return 0;
}
PetscErrorCode DMSetCoordinateDim(DM, PetscInt) { return 0; }
PetscErrorCode DMSetCoordinates(DM, Vec) { return 0; }
PetscErrorCode PetscObjectSetName(PetscObject, const char*) { return 0; }
MPI_Comm PetscObjectComm(PetscObject) { return 0; }
PetscErrorCode PetscViewerVTKOpen(MPI_Comm, const char*, PetscFileMode, PetscViewer* v) {
  *v = nullptr;
  return 0;
}
PetscErrorCode PetscViewerDestroy(PetscViewer*) { return 0; }
PetscErrorCode VecView(Vec, PetscViewer) { return 0; }
