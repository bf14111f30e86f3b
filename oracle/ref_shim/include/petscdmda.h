/*
 * Single-rank stand-in for the PETSc DMDA API, used only to compile the
 * reference M2C sources in place as a CPU oracle (test infrastructure).
 *
 * A DM describes one structured box of NX*NY*NZ nodes with `dof` doubles per
 * node and a ghost layer of width `s` on every side (DM_BOUNDARY_GHOSTED).
 * A local Vec holds the ghosted box; a global Vec holds the interior only.
 * DMDAVecGetArray returns the PETSc-style `double***` view indexed
 * [k][j][i*dof+p] with ghost indices -s..N+s-1. On one rank,
 * local->global copies (or adds) the interior, and global->local copies the
 * interior back, leaving ghost nodes outside the domain untouched, which is
 * what PETSc does for DM_BOUNDARY_GHOSTED.
 */
#ifndef M2C_ORACLE_PETSCDMDA_SHIM_H
#define M2C_ORACLE_PETSCDMDA_SHIM_H

#include <mpi.h>
#include <cstdio>

typedef int PetscErrorCode;
typedef int PetscInt;
typedef double PetscScalar;
typedef double PetscReal;
typedef enum { DM_BOUNDARY_NONE, DM_BOUNDARY_GHOSTED, DM_BOUNDARY_MIRROR, DM_BOUNDARY_PERIODIC,
               DM_BOUNDARY_TWIST } DMBoundaryType;
typedef enum { DMDA_STENCIL_STAR, DMDA_STENCIL_BOX } DMDAStencilType;
typedef enum { NOT_SET_VALUES, INSERT_VALUES, ADD_VALUES } InsertMode;
typedef enum { FILE_MODE_READ, FILE_MODE_WRITE, FILE_MODE_APPEND } PetscFileMode;

struct m2c_shim_dm;
struct m2c_shim_vec;
typedef m2c_shim_dm* DM;
typedef m2c_shim_vec* Vec;
typedef struct m2c_shim_viewer* PetscViewer;
typedef void* PetscObject;

#define PETSC_DECIDE (-1)
#define PETSC_NULL 0
#define CHKERRQ(ierr) do { if (ierr) return ierr; } while (0)

extern MPI_Comm PETSC_COMM_WORLD;

PetscErrorCode PetscInitialize(int*, char***, const char*, const char*);
PetscErrorCode PetscFinalize();
PetscErrorCode PetscPrintf(MPI_Comm, const char* fmt, ...);

PetscErrorCode DMDACreate3d(MPI_Comm, DMBoundaryType, DMBoundaryType, DMBoundaryType, DMDAStencilType,
                            PetscInt M, PetscInt N, PetscInt P, PetscInt m, PetscInt n, PetscInt p,
                            PetscInt dof, PetscInt s, const PetscInt*, const PetscInt*, const PetscInt*,
                            DM* da);
PetscErrorCode DMSetFromOptions(DM);
PetscErrorCode DMSetUp(DM);
PetscErrorCode DMDestroy(DM*);
PetscErrorCode DMDAGetInfo(DM, PetscInt* dim, PetscInt* M, PetscInt* N, PetscInt* P, PetscInt* m,
                           PetscInt* n, PetscInt* p, PetscInt* dof, PetscInt* s, DMBoundaryType* bx,
                           DMBoundaryType* by, DMBoundaryType* bz, DMDAStencilType* st);
PetscErrorCode DMDAGetCorners(DM, PetscInt* x, PetscInt* y, PetscInt* z, PetscInt* m, PetscInt* n,
                              PetscInt* p);
PetscErrorCode DMDAGetGhostCorners(DM, PetscInt* x, PetscInt* y, PetscInt* z, PetscInt* m, PetscInt* n,
                                   PetscInt* p);
PetscErrorCode DMCreateGlobalVector(DM, Vec*);
PetscErrorCode DMCreateLocalVector(DM, Vec*);
PetscErrorCode VecSet(Vec, PetscScalar);
PetscErrorCode VecDestroy(Vec*);
PetscErrorCode DMDAVecGetArray(DM, Vec, void* array);
PetscErrorCode DMDAVecRestoreArray(DM, Vec, void* array);
PetscErrorCode DMLocalToGlobal(DM, Vec l, InsertMode, Vec g);
PetscErrorCode DMGlobalToLocalBegin(DM, Vec g, InsertMode, Vec l);
PetscErrorCode DMGlobalToLocalEnd(DM, Vec g, InsertMode, Vec l);
PetscErrorCode DMSetCoordinateDim(DM, PetscInt);
PetscErrorCode DMSetCoordinates(DM, Vec);
PetscErrorCode PetscObjectSetName(PetscObject, const char*);
MPI_Comm PetscObjectComm(PetscObject);
PetscErrorCode PetscViewerVTKOpen(MPI_Comm, const char*, PetscFileMode, PetscViewer*);
PetscErrorCode PetscViewerDestroy(PetscViewer*);
PetscErrorCode VecView(Vec, PetscViewer);

#endif
