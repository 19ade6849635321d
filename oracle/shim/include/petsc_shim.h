/*
 * petsc_shim.h - the subset of the PETSc/MPI API that CIPHER's sources use,
 * re-declared so that the reference's own src/*.c compile unmodified into a
 * CPU oracle (test infrastructure; never part of the product).
 *
 * The DM is an explicit finite-volume mesh: points [0, ncells) are cells
 * (owned cells first, then ghosts), points [ncells, ncells+nfaces) are
 * interior faces in face order and the points after them are boundary faces.
 * Every cell carries `ndof` doubles.  Only the calls RHSFunction, PostStep,
 * SetUpProblem and the model code make are implemented; mesh creation,
 * adaptation, TS solving and viewers are stubs that return an error.
 */
#ifndef CIPHER_PETSC_SHIM_H
#define CIPHER_PETSC_SHIM_H

#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <stdint.h>
#include <math.h>

typedef int32_t PetscInt;
typedef int PetscMPIInt;
typedef double PetscReal;
typedef double PetscScalar;
typedef int PetscErrorCode;
typedef enum { PETSC_FALSE = 0, PETSC_TRUE = 1 } PetscBool;

#define PETSC_MAX_PATH_LEN 4096
#define PETSC_PI 3.14159265358979323846264338327950288419716939937510582
#define PETSC_DEFAULT (-2)
#define PETSC_DECIDE (-1)

#define CHKERRQ(e) do { if (e) return (e); } while (0)
#define PetscFunctionBegin do {} while (0)
#define PetscFunctionBeginUser do {} while (0)
#define PetscFunctionReturn(x) return (x)
#define PetscMalloc1(m, r) ((*(r) = malloc((size_t)(m) * sizeof(**(r)))) == NULL)

/* MPI */
typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
#define PETSC_COMM_WORLD 0
#define PETSC_COMM_SELF 1
#define MPI_CHAR 1
#define MPIU_SCALAR 2
#define MPI_LAND 1
#define MPI_LOR 2
#define MPI_SUM 3
#define MPI_REPLACE 4
#define MPI_IN_PLACE ((void *)1)
int MPI_Comm_rank(MPI_Comm, int *);
int MPI_Comm_size(MPI_Comm, int *);
int MPI_Allreduce(const void *, void *, int, MPI_Datatype, MPI_Op, MPI_Comm);

/* opaque objects */
typedef struct _p_DM *DM;
typedef struct _p_Vec *Vec;
typedef struct _p_TS *TS;
typedef struct _p_IS *IS;
typedef struct _p_DMLabel *DMLabel;
typedef struct _p_PetscSection *PetscSection;
typedef struct _p_PetscSF *PetscSF;
typedef struct _p_PetscViewer *PetscViewer;
typedef struct _p_PetscFE *PetscFE;
typedef struct _p_TSAdapt *TSAdapt;
typedef struct _p_PetscObject *PetscObject;
typedef const char *DMType;
typedef const char *TSType;
typedef const char *TSAdaptType;

typedef struct { PetscInt rank, index; } PetscSFNode;
typedef struct { PetscReal centroid[3]; PetscReal volume; } PetscFVCellGeom;

typedef enum { INSERT_VALUES = 1, ADD_VALUES = 2 } InsertMode;
typedef enum { PETSC_COPY_VALUES = 0, PETSC_OWN_POINTER = 1, PETSC_USE_POINTER = 2 } PetscCopyMode;
typedef enum { DM_COPY_LABELS_REPLACE = 0, DM_COPY_LABELS_KEEP = 1, DM_COPY_LABELS_FAIL = 2 } DMCopyLabelsMode;
typedef enum { TS_EXACTFINALTIME_UNSPECIFIED = 0, TS_EXACTFINALTIME_STEPOVER = 1,
               TS_EXACTFINALTIME_INTERPOLATE = 2, TS_EXACTFINALTIME_MATCHSTEP = 3 } TSExactFinalTimeOption;
typedef enum { PETSC_VIEWER_DEFAULT = 0, PETSC_VIEWER_VTK_VTU = 1 } PetscViewerFormat;
typedef enum { FILE_MODE_READ = 0, FILE_MODE_WRITE = 1 } PetscFileMode;
enum { DM_ADAPT_DETERMINE = -1, DM_ADAPT_KEEP = 0, DM_ADAPT_REFINE = 1, DM_ADAPT_COARSEN = 2 };

#define DMPLEX "plex"
#define DMP4EST "p4est"
#define DMP8EST "p8est"
#define TSRK "rk"
#define TSADAPTDSP "dsp"

/* init / options / printing */
PetscErrorCode PetscInitialize(int *, char ***, const char *, const char *);
PetscErrorCode PetscFinalize(void);
PetscErrorCode PetscPrintf(MPI_Comm, const char *, ...);
PetscErrorCode PetscOptionsInsertString(void *, const char *);
PetscErrorCode PetscOptionsGetString(void *, const char *, const char *, char *, size_t, PetscBool *);
PetscErrorCode PetscObjectSetName(PetscObject, const char *);
MPI_Comm PetscObjectComm(PetscObject);

/* Vec */
PetscErrorCode VecGetArray(Vec, PetscScalar **);
PetscErrorCode VecRestoreArray(Vec, PetscScalar **);
PetscErrorCode VecGetArrayRead(Vec, const PetscScalar **);
PetscErrorCode VecRestoreArrayRead(Vec, const PetscScalar **);
PetscErrorCode VecZeroEntries(Vec);
PetscErrorCode VecCopy(Vec, Vec);
PetscErrorCode VecDestroy(Vec *);
PetscErrorCode VecGetDM(Vec, DM *);
PetscErrorCode VecView(Vec, PetscViewer);

/* DM */
PetscErrorCode DMCreate(MPI_Comm, DM *);
PetscErrorCode DMSetType(DM, DMType);
PetscErrorCode DMSetFromOptions(DM);
PetscErrorCode DMSetUp(DM);
PetscErrorCode DMConvert(DM, DMType, DM *);
PetscErrorCode DMLocalizeCoordinates(DM);
PetscErrorCode DMDestroy(DM *);
PetscErrorCode DMClone(DM, DM *);
PetscErrorCode DMSetField(DM, PetscInt, DMLabel, PetscObject);
PetscErrorCode DMCreateDS(DM);
PetscErrorCode DMCopyDisc(DM, DM);
PetscErrorCode DMGetSection(DM, PetscSection *);
PetscErrorCode DMGetGlobalSection(DM, PetscSection *);
PetscErrorCode DMCreateGlobalVector(DM, Vec *);
PetscErrorCode DMGetLocalVector(DM, Vec *);
PetscErrorCode DMRestoreLocalVector(DM, Vec *);
PetscErrorCode DMGetGlobalVector(DM, Vec *);
PetscErrorCode DMRestoreGlobalVector(DM, Vec *);
PetscErrorCode DMGlobalToLocalBegin(DM, Vec, InsertMode, Vec);
PetscErrorCode DMGlobalToLocalEnd(DM, Vec, InsertMode, Vec);
PetscErrorCode DMCreateLabel(DM, const char *);
PetscErrorCode DMGetLabel(DM, const char *, DMLabel *);
PetscErrorCode DMSetLabelValue(DM, const char *, PetscInt, PetscInt);
PetscErrorCode DMGetLabelValue(DM, const char *, PetscInt, PetscInt *);
PetscErrorCode DMCopyLabels(DM, DM, PetscCopyMode, PetscBool, DMCopyLabelsMode);
PetscErrorCode DMAdaptLabel(DM, DMLabel, DM *);
PetscErrorCode DMForestSetTopology(DM, const char *);
PetscErrorCode DMForestSetInitialRefinement(DM, PetscInt);
PetscErrorCode DMForestSetMaximumRefinement(DM, PetscInt);
PetscErrorCode DMForestSetMinimumRefinement(DM, PetscInt);
PetscErrorCode DMForestSetPartitionOverlap(DM, PetscInt);
PetscErrorCode DMForestSetAdaptivityForest(DM, DM);
PetscErrorCode DMForestTransferVec(DM, Vec, DM, Vec, PetscBool, PetscReal);

/* DMPlex */
PetscErrorCode DMPlexGetHeightStratum(DM, PetscInt, PetscInt *, PetscInt *);
PetscErrorCode DMPlexGetConeSize(DM, PetscInt, PetscInt *);
PetscErrorCode DMPlexGetCone(DM, PetscInt, const PetscInt **);
PetscErrorCode DMPlexGetSupportSize(DM, PetscInt, PetscInt *);
PetscErrorCode DMPlexGetSupport(DM, PetscInt, const PetscInt **);
PetscErrorCode DMPlexGetTreeChildren(DM, PetscInt, PetscInt *, const PetscInt **);
PetscErrorCode DMPlexPointLocalRef(DM, PetscInt, PetscScalar *, void *);
PetscErrorCode DMPlexPointGlobalRef(DM, PetscInt, PetscScalar *, void *);
PetscErrorCode DMPlexPointLocalRead(DM, PetscInt, const PetscScalar *, void *);
PetscErrorCode DMPlexComputeCellGeometryFVM(DM, PetscInt, PetscReal *, PetscReal *, PetscReal *);
PetscErrorCode DMPlexGetDataFVM(DM, void *, Vec *, Vec *, DM *);

/* sections, labels, index sets */
PetscErrorCode PetscSectionGetDof(PetscSection, PetscInt, PetscInt *);
PetscErrorCode DMLabelCreate(MPI_Comm, const char *, DMLabel *);
PetscErrorCode DMLabelSetDefaultValue(DMLabel, PetscInt);
PetscErrorCode DMLabelSetValue(DMLabel, PetscInt, PetscInt);
PetscErrorCode DMLabelGetValue(DMLabel, PetscInt, PetscInt *);
PetscErrorCode DMLabelGetStratumIS(DMLabel, PetscInt, IS *);
PetscErrorCode ISGetLocalSize(IS, PetscInt *);
PetscErrorCode ISGetIndices(IS, const PetscInt **);
PetscErrorCode ISRestoreIndices(IS, const PetscInt **);
PetscErrorCode ISGetMinMax(IS, PetscInt *, PetscInt *);
PetscErrorCode ISDestroy(IS *);

/* star forest */
PetscErrorCode PetscSFCreate(MPI_Comm, PetscSF *);
PetscErrorCode PetscSFSetFromOptions(PetscSF);
PetscErrorCode PetscSFSetGraph(PetscSF, PetscInt, PetscInt, PetscInt *, PetscCopyMode, PetscSFNode *, PetscCopyMode);
PetscErrorCode PetscSFSetUp(PetscSF);
PetscErrorCode PetscSFDestroy(PetscSF *);
PetscErrorCode PetscSFReduceBegin(PetscSF, MPI_Datatype, const void *, void *, MPI_Op);
PetscErrorCode PetscSFReduceEnd(PetscSF, MPI_Datatype, const void *, void *, MPI_Op);
PetscErrorCode PetscSFBcastBegin(PetscSF, MPI_Datatype, const void *, void *, MPI_Op);
PetscErrorCode PetscSFBcastEnd(PetscSF, MPI_Datatype, const void *, void *, MPI_Op);

/* FE (discretisation objects) */
PetscErrorCode PetscFECreateDefault(MPI_Comm, PetscInt, PetscInt, PetscBool, const char *, PetscInt, PetscFE *);
PetscErrorCode PetscFEDestroy(PetscFE *);

/* viewers */
PetscErrorCode PetscViewerVTKOpen(MPI_Comm, const char *, PetscFileMode, PetscViewer *);
PetscErrorCode PetscViewerPushFormat(PetscViewer, PetscViewerFormat);
PetscErrorCode PetscViewerDestroy(PetscViewer *);

/* TS */
PetscErrorCode TSCreate(MPI_Comm, TS *);
PetscErrorCode TSSetType(TS, TSType);
PetscErrorCode TSSetDM(TS, DM);
PetscErrorCode TSSetApplicationContext(TS, void *);
PetscErrorCode TSGetApplicationContext(TS, void *);
PetscErrorCode TSSetRHSFunction(TS, Vec, PetscErrorCode (*)(TS, PetscReal, Vec, Vec, void *), void *);
PetscErrorCode TSSetPostStep(TS, PetscErrorCode (*)(TS));
PetscErrorCode TSGetAdapt(TS, TSAdapt *);
PetscErrorCode TSAdaptSetType(TSAdapt, TSAdaptType);
PetscErrorCode TSAdaptSetStepLimits(TSAdapt, PetscReal, PetscReal);
PetscErrorCode TSSetTolerances(TS, PetscReal, Vec, PetscReal, Vec);
PetscErrorCode TSSetFromOptions(TS);
PetscErrorCode TSGetSolution(TS, Vec *);
PetscErrorCode TSSetSolution(TS, Vec);
PetscErrorCode TSGetTime(TS, PetscReal *);
PetscErrorCode TSSetTime(TS, PetscReal);
PetscErrorCode TSGetTimeStep(TS, PetscReal *);
PetscErrorCode TSSetTimeStep(TS, PetscReal);
PetscErrorCode TSGetStepNumber(TS, PetscInt *);
PetscErrorCode TSSetStepNumber(TS, PetscInt);
PetscErrorCode TSGetSolveTime(TS, PetscReal *);
PetscErrorCode TSSetMaxSteps(TS, PetscInt);
PetscErrorCode TSSetMaxTime(TS, PetscReal);
PetscErrorCode TSSetExactFinalTime(TS, TSExactFinalTimeOption);
PetscErrorCode TSSolve(TS, Vec);
PetscErrorCode TSDestroy(TS *);

#endif /* CIPHER_PETSC_SHIM_H */
