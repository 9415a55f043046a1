/*
 * ref_driver.c -- C entry points of the reference build for the tests.
 * TEST INFRASTRUCTURE ONLY: compiled into oracle/_ref/libpastix_ref.so next to
 * the reference's own sources, never into the product.
 *
 * A handle wraps one pastix_data_t of the reference and one SpM descriptor.
 * The tests set iparm / dparm through the arrays the handle exposes, give the
 * matrix (CSC, 0-based), run the reference's analysis with a grid nested
 * dissection (order/order_grids.c:307, as example/ordering_grid.c does) or a
 * caller permutation (PastixOrderPersonal), and read back what the product
 * must reproduce: the ordering, the SolverMatrix structure (blend/solver.h:
 * 141-279), the factors in a normalized per-blok layout, the static-pivot
 * count, solutions and refinement results.
 */
#include "common.h"
#include "blend/solver.h"
#include "symbol/symbol.h"
#include "pastix/order.h"

#include <string.h>

typedef struct ref_handle_s {
    pastix_data_t *pd;
    pastix_int_t   iparm[IPARM_SIZE];
    double         dparm[DPARM_SIZE];
    spmatrix_t     spm;
    int            has_spm;
} ref_handle_t;

ref_handle_t *ref_new( void )
{
    ref_handle_t *h = calloc( 1, sizeof( *h ) );
    pastixInitParam( h->iparm, h->dparm );
    h->iparm[IPARM_VERBOSE] = PastixVerboseNot;
    return h;
}

pastix_int_t *ref_iparm( ref_handle_t *h ) { return h->iparm; }
double       *ref_dparm( ref_handle_t *h ) { return h->dparm; }

int ref_init( ref_handle_t *h )
{
    pastixInit( &h->pd, MPI_COMM_WORLD, h->iparm, h->dparm );
    return h->pd ? PASTIX_SUCCESS : PASTIX_ERR_INTERNAL;
}

void ref_free( ref_handle_t *h )
{
    if ( h == NULL ) {
        return;
    }
    if ( h->pd ) {
        pastixFinalize( &h->pd );
    }
    if ( h->has_spm ) {
        spmExit( &h->spm );
    }
    free( h );
}

/* CSC matrix, 0-based, copied.  mtxtype: SpmGeneral / SpmSymmetric (lower
 * triangle stored).  values may be NULL (pattern only). */
int ref_set_matrix( ref_handle_t *h, pastix_int_t n, const pastix_int_t *colptr, const pastix_int_t *rowptr,
                    const double *values, int mtxtype, pastix_int_t dof )
{
    if ( h->has_spm ) {
        spmExit( &h->spm );
    }
    spmatrix_t *s = &h->spm;
    spmInit( s );
    s->mtxtype = (spm_mtxtype_t)mtxtype;
    s->flttype = values ? SpmDouble : SpmPattern;
    s->fmttype = SpmCSC;
    s->baseval = 0;
    s->n       = n;
    s->nnz     = colptr[n];
    s->dof     = dof;
    s->colptr  = malloc( ( n + 1 ) * sizeof( pastix_int_t ) );
    s->rowptr  = malloc( ( s->nnz ? s->nnz : 1 ) * sizeof( pastix_int_t ) );
    memcpy( s->colptr, colptr, ( n + 1 ) * sizeof( pastix_int_t ) );
    memcpy( s->rowptr, rowptr, s->nnz * sizeof( pastix_int_t ) );
    if ( values ) {
        size_t nv = (size_t)s->nnz * dof * dof;
        s->values = malloc( ( nv ? nv : 1 ) * sizeof( double ) );
        memcpy( s->values, values, nv * sizeof( double ) );
    }
    spmUpdateComputedFields( s );
    h->has_spm = 1;
    return PASTIX_SUCCESS;
}

/* New values for the same pattern (refactorization). */
int ref_set_values( ref_handle_t *h, const double *values )
{
    if ( !h->has_spm || h->spm.values == NULL ) {
        return PASTIX_ERR_BADPARAMETER;
    }
    memcpy( h->spm.values, values, (size_t)h->spm.nnzexp * sizeof( double ) );
    return PASTIX_SUCCESS;
}

/*
 * The reference's analysis: ordering, symbolic factorization, reordering and
 * blend (blend/pastix_task_analyze.c:53 does the same four steps).  With
 * nx > 0 the ordering is pastixOrderGrid(nx, ny, nz); otherwise `perm`
 * (permtab, 0-based, size n) is given as a personal ordering whose
 * supernodes the reference finds itself.
 */
int ref_analyze( ref_handle_t *h, pastix_int_t nx, pastix_int_t ny, pastix_int_t nz, const pastix_int_t *perm )
{
    pastix_order_t *ord = NULL;
    int             rc;
    if ( !h->has_spm || !h->pd ) {
        return PASTIX_ERR_BADPARAMETER;
    }
    if ( nx > 0 ) {
        ord = malloc( sizeof( pastix_order_t ) );
        rc  = pastixOrderGrid( &ord, nx, ny, nz );
        if ( rc != PASTIX_SUCCESS ) {
            return rc;
        }
    }
    else if ( perm ) {
        pastix_int_t n = h->spm.n, i;
        ord = malloc( sizeof( pastix_order_t ) );
        pastixOrderAlloc( ord, n, 0 );
        for ( i = 0; i < n; i++ ) {
            ord->permtab[i]       = perm[i];
            ord->peritab[perm[i]] = i;
        }
    }
    if ( ord ) {
        h->iparm[IPARM_ORDERING] = PastixOrderPersonal;
    }
    rc = pastix_subtask_order( h->pd, &h->spm, ord );
    if ( ord ) {
        pastixOrderExit( ord );
        free( ord );
    }
    if ( rc != PASTIX_SUCCESS ) return rc;
    rc = pastix_subtask_symbfact( h->pd );
    if ( rc != PASTIX_SUCCESS ) return rc;
    rc = pastix_subtask_reordering( h->pd );
    if ( rc != PASTIX_SUCCESS ) return rc;
    return pastix_subtask_blend( h->pd );
}

/* sizes[0..5] = n (columns after dof expansion), cblknbr, bloknbr, coefnbr,
 * order cblknbr, order vertnbr */
int ref_sizes( ref_handle_t *h, pastix_int_t *sizes )
{
    const SolverMatrix *s = h->pd ? h->pd->solvmatr : NULL;
    if ( s == NULL ) {
        return PASTIX_ERR_BADPARAMETER;
    }
    sizes[0] = s->nodenbr;
    sizes[1] = s->cblknbr;
    sizes[2] = s->bloknbr;
    sizes[3] = s->coefnbr;
    sizes[4] = h->pd->ordemesh ? h->pd->ordemesh->cblknbr : 0;
    sizes[5] = h->pd->ordemesh ? h->pd->ordemesh->vertnbr : 0;
    return PASTIX_SUCCESS;
}

/* The ordering after the analysis (level order and reordering included):
 * permtab / peritab (vertnbr), rangtab (cblknbr + 1), treetab (cblknbr). */
int ref_get_order( ref_handle_t *h, pastix_int_t *permtab, pastix_int_t *peritab, pastix_int_t *rangtab,
                   pastix_int_t *treetab )
{
    const pastix_order_t *o = h->pd ? h->pd->ordemesh : NULL;
    pastix_int_t          b;
    if ( o == NULL ) {
        return PASTIX_ERR_BADPARAMETER;
    }
    b = o->baseval;
    for ( pastix_int_t i = 0; i < o->vertnbr; i++ ) {
        permtab[i] = o->permtab[i] - b;
        peritab[i] = o->peritab[i] - b;
    }
    for ( pastix_int_t k = 0; k <= o->cblknbr; k++ ) rangtab[k] = o->rangtab[k] - b;
    if ( treetab && o->treetab ) {
        for ( pastix_int_t k = 0; k < o->cblknbr; k++ ) treetab[k] = o->treetab[k] < 0 ? -1 : o->treetab[k] - b;
    }
    return PASTIX_SUCCESS;
}

/* SolverMatrix structure: per cblk first / last column, first blok, stride,
 * type flags; per blok first / last row, facing cblk. */
int ref_get_solver( ref_handle_t *h, pastix_int_t *cb_fcol, pastix_int_t *cb_lcol, pastix_int_t *cb_fblok,
                    pastix_int_t *cb_stride, pastix_int_t *cb_type, pastix_int_t *bk_frow, pastix_int_t *bk_lrow,
                    pastix_int_t *bk_fcblk )
{
    const SolverMatrix *s = h->pd ? h->pd->solvmatr : NULL;
    if ( s == NULL ) {
        return PASTIX_ERR_BADPARAMETER;
    }
    for ( pastix_int_t k = 0; k < s->cblknbr; k++ ) {
        const SolverCblk *c = s->cblktab + k;
        cb_fcol[k]   = c->fcolnum;
        cb_lcol[k]   = c->lcolnum;
        cb_fblok[k]  = c->fblokptr - s->bloktab;
        cb_stride[k] = c->stride;
        cb_type[k]   = c->cblktype;
    }
    cb_fblok[s->cblknbr] = s->bloknbr;
    for ( pastix_int_t b = 0; b < s->bloknbr; b++ ) {
        bk_frow[b]  = s->bloktab[b].frownum;
        bk_lrow[b]  = s->bloktab[b].lrownum;
        bk_fcblk[b] = s->bloktab[b].fcblknm;
    }
    return PASTIX_SUCCESS;
}

int ref_numfact( ref_handle_t *h )
{
    return pastix_task_numfact( h->pd, &h->spm );
}

/*
 * Factors after ref_numfact in a normalized per-blok layout: blok b of cblk k
 * (nrows x width) at dst + coefind[b], column-major with leading dimension
 * nrows, whatever the reference's own layout of the cblk (1D: one panel with
 * leading dimension stride; 2D: one tile per blok).  side 0: L (lcoeftab),
 * 1: U (ucoeftab, LU only).  FP32 factors (IPARM_MIXED) are widened.
 */
int ref_get_coef( ref_handle_t *h, int side, const pastix_int_t *coefind, double *dst )
{
    const SolverMatrix *s = h->pd ? h->pd->solvmatr : NULL;
    if ( s == NULL ) {
        return PASTIX_ERR_BADPARAMETER;
    }
    const int single = ( s->flttype == PastixFloat );
    for ( pastix_int_t k = 0; k < s->cblknbr; k++ ) {
        const SolverCblk *c    = s->cblktab + k;
        const void       *src  = side ? c->ucoeftab : c->lcoeftab;
        const int         is2d = ( c->cblktype & CBLK_LAYOUT_2D ) != 0;
        pastix_int_t      nc   = c->lcolnum - c->fcolnum + 1;
        if ( src == NULL ) {
            return PASTIX_ERR_BADPARAMETER;
        }
        for ( const SolverBlok *b = c->fblokptr; b < c[1].fblokptr; b++ ) {
            pastix_int_t nr = b->lrownum - b->frownum + 1;
            pastix_int_t ld = is2d ? nr : c->stride;
            double      *d  = dst + coefind[b - s->bloktab];
            for ( pastix_int_t j = 0; j < nc; j++ ) {
                for ( pastix_int_t i = 0; i < nr; i++ ) {
                    pastix_int_t e = b->coefind + j * ld + i;
                    d[j * nr + i]  = single ? (double)( (const float *)src )[e] : ( (const double *)src )[e];
                }
            }
        }
    }
    return PASTIX_SUCCESS;
}

/* A X = B in place (pastix_task_solve, sopalin/pastix_task_solve.c:758). */
int ref_solve( ref_handle_t *h, pastix_int_t nrhs, double *b, pastix_int_t ldb )
{
    return pastix_task_solve( h->pd, h->spm.nexp, nrhs, b, ldb );
}

/* Iterative refinement of x (pastix_task_refine, refinement/pastix_task_refine.c:236). */
int ref_refine( ref_handle_t *h, pastix_int_t nrhs, double *b, pastix_int_t ldb, double *x, pastix_int_t ldx )
{
    return pastix_task_refine( h->pd, h->spm.nexp, nrhs, b, ldb, x, ldx );
}

/*
 * Distance between the reference's factors and factors stored in the product's
 * panel layout (cblk k: one column-major panel of stride x width at
 * cb_coef[k], blok b starting at row bk_rowoff[b]) for the same structure,
 * without a second copy of the factors: out[0] = sum (ref - P)^2,
 * out[1] = sum ref^2.  mask_upper skips the strict upper triangle of the
 * diagonal blocks (unused by LL^T).  P holds doubles, or floats if single.
 */
int ref_compare_panels( ref_handle_t *h, int side, const void *P, int single, const pastix_int_t *cb_coef,
                        const pastix_int_t *cb_stride, const pastix_int_t *bk_rowoff, int mask_upper, double *out )
{
    const SolverMatrix *s = h->pd ? h->pd->solvmatr : NULL;
    double              d2 = 0.0, r2 = 0.0;
    if ( s == NULL ) {
        return PASTIX_ERR_BADPARAMETER;
    }
    const int rsingle = ( s->flttype == PastixFloat );
    #pragma omp parallel for reduction(+:d2,r2) schedule(dynamic, 16)
    for ( pastix_int_t k = 0; k < s->cblknbr; k++ ) {
        const SolverCblk *c    = s->cblktab + k;
        const void       *src  = side ? c->ucoeftab : c->lcoeftab;
        const int         is2d = ( c->cblktype & CBLK_LAYOUT_2D ) != 0;
        pastix_int_t      nc   = c->lcolnum - c->fcolnum + 1;
        if ( src == NULL ) {
            continue;
        }
        for ( const SolverBlok *b = c->fblokptr; b < c[1].fblokptr; b++ ) {
            pastix_int_t nr   = b->lrownum - b->frownum + 1;
            pastix_int_t ld   = is2d ? nr : c->stride;
            pastix_int_t bi   = b - s->bloktab;
            int          diag = ( b == c->fblokptr );
            for ( pastix_int_t j = 0; j < nc; j++ ) {
                for ( pastix_int_t i = ( diag && mask_upper ) ? j : 0; i < nr; i++ ) {
                    pastix_int_t e  = b->coefind + j * ld + i;
                    pastix_int_t q  = cb_coef[k] + bk_rowoff[bi] + i + j * cb_stride[k];
                    double       rv = rsingle ? (double)( (const float *)src )[e] : ( (const double *)src )[e];
                    double       pv = single ? (double)( (const float *)P )[q] : ( (const double *)P )[q];
                    d2 += ( rv - pv ) * ( rv - pv );
                    r2 += rv * rv;
                }
            }
        }
    }
    out[0] = d2;
    out[1] = r2;
    return PASTIX_SUCCESS;
}
