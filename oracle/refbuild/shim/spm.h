/*
 * spm.h -- minimal SpM interface for compiling the reference's sources as the
 * oracle.  TEST INFRASTRUCTURE ONLY.
 *
 * PaStiX takes its matrices from the SpM library, a git submodule that is not
 * part of the reference checkout.  This header restates the part of SpM's
 * interface that the reference's ordering, symbolic, blend and numerical code
 * uses (the descriptor's fields, the enumerations and the dozen routines called
 * by graph/graph.c, sopalin/pastix_task_sopalin.c and sopalin/pastix.c);
 * spm_min.c implements the routines for one process and centralized CSC
 * matrices, which is all the oracle runs.
 */
#ifndef ORACLE_SPM_H
#define ORACLE_SPM_H

#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <complex.h>
#include <inttypes.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int64_t spm_int_t;          /* PaStiX is built with 64-bit integers here */
typedef uintptr_t SPM_Comm;         /* no MPI: same placeholder as PASTIX_Comm    */
typedef float _Complex  spm_complex32_t;
typedef double _Complex spm_complex64_t;

#define SPM_SUCCESS            0
#define SPM_ERR_UNKNOWN        1
#define SPM_ERR_ALLOC          2
#define SPM_ERR_NOTIMPLEMENTED 3
#define SPM_ERR_OUTOFMEMORY    4
#define SPM_ERR_BADPARAMETER   7
#define SPM_ERR_FILE           8

typedef enum spm_coeftype_e {
    SpmPattern = 0, SpmFloat = 2, SpmDouble = 3, SpmComplex32 = 4, SpmComplex64 = 5
} spm_coeftype_t;

typedef enum spm_mtxtype_e {
    SpmGeneral = 111, SpmSymmetric = 112, SpmHermitian = 113
} spm_mtxtype_t;

typedef enum spm_fmttype_e { SpmCSC = 0, SpmCSR = 1, SpmIJV = 2 } spm_fmttype_t;

typedef enum spm_layout_e { SpmRowMajor = 101, SpmColMajor = 102 } spm_layout_t;

typedef enum spm_normtype_e {
    SpmOneNorm = 171, SpmFrobeniusNorm = 174, SpmInfNorm = 175, SpmMaxNorm = 177
} spm_normtype_t;

typedef enum spm_rhstype_e { SpmRhsOne, SpmRhsI, SpmRhsRndX, SpmRhsRndB } spm_rhstype_t;

typedef enum spm_driver_e {
    SpmDriverRSA, SpmDriverHB, SpmDriverIJV, SpmDriverMM, SpmDriverLaplacian,
    SpmDriverXLaplacian, SpmDriverGraph, SpmDriverSPM
} spm_driver_t;

typedef struct spmatrix_s {
    spm_mtxtype_t  mtxtype;
    spm_coeftype_t flttype;
    spm_fmttype_t  fmttype;
    spm_int_t      baseval;
    spm_int_t      gN, n, gnnz, nnz;
    spm_int_t      gNexp, nexp, gnnzexp, nnzexp;
    spm_int_t      dof;       /* > 0: constant dof per vertex; < 1: variable (dofs) */
    spm_int_t     *dofs;
    spm_layout_t   layout;
    spm_int_t     *colptr;
    spm_int_t     *rowptr;
    spm_int_t     *loc2glob;
    void          *values;
    spm_int_t     *glob2loc;
    int            clustnum, clustnbr;
    SPM_Comm       comm;
    int            replicated;
} spmatrix_t;

void      spmInit( spmatrix_t *spm );
void      spmInitDist( spmatrix_t *spm, SPM_Comm comm );
void      spmExit( spmatrix_t *spm );
void      spmBase( spmatrix_t *spm, int baseval );
spm_int_t spmFindBase( const spmatrix_t *spm );
void      spmCopy( const spmatrix_t *spmin, spmatrix_t *spmout );
int       spmSort( spmatrix_t *spm );
spm_int_t spmSymmetrize( spmatrix_t *spm );
void      spmUpdateComputedFields( spmatrix_t *spm );
int       spmConvert( int ofmttype, spmatrix_t *ospm );
double    spmNorm( spm_normtype_t ntype, const spmatrix_t *spm );
int       spmExpand( const spmatrix_t *spm_in, spmatrix_t *spm_out );
int       spmScatter( spmatrix_t *spm_scattered, int root, const spmatrix_t *opt_spm_gathered,
                      spm_int_t opt_n, const spm_int_t *opt_loc2glob, int opt_distByColumn, SPM_Comm opt_comm );
int       spmGather( const spmatrix_t *spm_scattered, int root, spmatrix_t *opt_spm_gathered );
int       spmLoad( spmatrix_t *spm, const char *filename );
int       spmSave( const spmatrix_t *spm, const char *filename );
spm_int_t *spm_get_glob2loc( spmatrix_t *spm );

#ifdef __cplusplus
}
#endif
#endif
