/*
 * spm_min.c -- the SpM routines the reference's sources call, for one process
 * and centralized CSC matrices.  TEST INFRASTRUCTURE ONLY (oracle build).
 *
 * Semantics follow how the reference uses them: graph/graph.c copies the
 * user's matrix into a pattern graph (spmCopy, spmConvert), mirrors the
 * stored triangle of a symmetric matrix (spmSymmetrize), sorts each column
 * (spmSort) and rebases it (spmBase); sopalin/pastix_task_sopalin.c:118 takes
 * the Frobenius norm of the whole matrix (spmNorm; the mirrored triangle of a
 * symmetric matrix counts twice).  Distribution (spmScatter / spmGather) and
 * file I/O are not needed and report SPM_ERR_NOTIMPLEMENTED.
 */
#include "spm.h"

#include <math.h>
#include <string.h>

static size_t flt_size( spm_coeftype_t t )
{
    switch ( t ) {
    case SpmFloat:     return 4;
    case SpmDouble:    return 8;
    case SpmComplex32: return 8;
    case SpmComplex64: return 16;
    default:           return 0;
    }
}

static spm_int_t dof_of( const spmatrix_t *spm, spm_int_t j )
{
    if ( spm->dof > 0 ) {
        return spm->dof;
    }
    return spm->dofs[j + 1] - spm->dofs[j];
}

void spmInitDist( spmatrix_t *spm, SPM_Comm comm )
{
    memset( spm, 0, sizeof( *spm ) );
    spm->mtxtype    = SpmGeneral;
    spm->flttype    = SpmDouble;
    spm->fmttype    = SpmCSC;
    spm->dof        = 1;
    spm->layout     = SpmColMajor;
    spm->clustnum   = 0;
    spm->clustnbr   = 1;
    spm->comm       = comm;
    spm->replicated = -1;
}

void spmInit( spmatrix_t *spm ) { spmInitDist( spm, 0 ); }

void spmExit( spmatrix_t *spm )
{
    free( spm->colptr );
    free( spm->rowptr );
    free( spm->loc2glob );
    free( spm->glob2loc );
    free( spm->values );
    free( spm->dofs );
    spm->colptr = spm->rowptr = spm->loc2glob = spm->glob2loc = spm->dofs = NULL;
    spm->values = NULL;
}

spm_int_t spmFindBase( const spmatrix_t *spm )
{
    spm_int_t b = spm->colptr[0];
    for ( spm_int_t e = 0; e < spm->nnz && b > 0; e++ ) {
        if ( spm->rowptr[e] < b ) {
            b = spm->rowptr[e];
        }
    }
    return b > 0 ? 1 : 0;
}

void spmBase( spmatrix_t *spm, int baseval )
{
    spm_int_t d = (spm_int_t)baseval - spm->baseval;
    if ( d == 0 ) {
        return;
    }
    for ( spm_int_t j = 0; j <= spm->n; j++ ) spm->colptr[j] += d;
    for ( spm_int_t e = 0; e < spm->nnz; e++ ) spm->rowptr[e] += d;
    if ( spm->loc2glob ) {
        for ( spm_int_t j = 0; j < spm->n; j++ ) spm->loc2glob[j] += d;
    }
    if ( spm->dofs ) {
        for ( spm_int_t j = 0; j <= spm->gN; j++ ) spm->dofs[j] += d;
    }
    spm->baseval = baseval;
}

/* number of stored scalar values (dof blocks expanded) */
static spm_int_t value_count( const spmatrix_t *spm )
{
    if ( spm->dof > 0 ) {
        return spm->nnz * spm->dof * spm->dof;
    }
    spm_int_t cnt = 0;
    for ( spm_int_t j = 0; j < spm->n; j++ ) {
        for ( spm_int_t e = spm->colptr[j] - spm->baseval; e < spm->colptr[j + 1] - spm->baseval; e++ ) {
            cnt += dof_of( spm, j ) * dof_of( spm, spm->rowptr[e] - spm->baseval );
        }
    }
    return cnt;
}

static void *dup_bytes( const void *src, size_t bytes )
{
    if ( src == NULL ) {
        return NULL;
    }
    void *p = malloc( bytes ? bytes : 1 );
    memcpy( p, src, bytes );
    return p;
}

void spmCopy( const spmatrix_t *in, spmatrix_t *out )
{
    memcpy( out, in, sizeof( *out ) );
    out->colptr   = dup_bytes( in->colptr, ( in->n + 1 ) * sizeof( spm_int_t ) );
    out->rowptr   = dup_bytes( in->rowptr, in->nnz * sizeof( spm_int_t ) );
    out->loc2glob = dup_bytes( in->loc2glob, in->n * sizeof( spm_int_t ) );
    out->glob2loc = dup_bytes( in->glob2loc, in->gN * sizeof( spm_int_t ) );
    out->dofs     = dup_bytes( in->dofs, ( in->gN + 1 ) * sizeof( spm_int_t ) );
    out->values   = ( in->flttype == SpmPattern || in->values == NULL )
                  ? NULL : dup_bytes( in->values, value_count( in ) * flt_size( in->flttype ) );
}

int spmConvert( int ofmttype, spmatrix_t *spm )
{
    return ( ofmttype == (int)spm->fmttype ) ? SPM_SUCCESS : SPM_ERR_NOTIMPLEMENTED;
}

static int cmp_int( const void *a, const void *b )
{
    spm_int_t x = *(const spm_int_t *)a, y = *(const spm_int_t *)b;
    return ( x > y ) - ( x < y );
}

/* row indices of every column in increasing order (values follow for scalar double) */
int spmSort( spmatrix_t *spm )
{
    const spm_int_t b = spm->baseval;
    for ( spm_int_t j = 0; j < spm->n; j++ ) {
        spm_int_t e0 = spm->colptr[j] - b, e1 = spm->colptr[j + 1] - b;
        if ( spm->values == NULL || spm->flttype == SpmPattern ) {
            qsort( spm->rowptr + e0, e1 - e0, sizeof( spm_int_t ), cmp_int );
            continue;
        }
        if ( spm->flttype != SpmDouble || spm->dof != 1 ) {
            return SPM_ERR_NOTIMPLEMENTED;
        }
        double *v = (double *)spm->values;
        for ( spm_int_t i = e0 + 1; i < e1; i++ ) { /* insertion sort, columns are short */
            spm_int_t r = spm->rowptr[i];
            double    x = v[i];
            spm_int_t k = i - 1;
            while ( k >= e0 && spm->rowptr[k] > r ) {
                spm->rowptr[k + 1] = spm->rowptr[k];
                v[k + 1]           = v[k];
                k--;
            }
            spm->rowptr[k + 1] = r;
            v[k + 1]           = x;
        }
    }
    return SPM_SUCCESS;
}

/* Adds (j, i) for every stored (i, j) whose mirror is absent; returns the count
 * added.  Pattern only: the oracle calls it on graphs. */
spm_int_t spmSymmetrize( spmatrix_t *spm )
{
    const spm_int_t n = spm->n, b = spm->baseval;
    if ( spm->values != NULL && spm->flttype != SpmPattern ) {
        return -1;
    }
    spm_int_t *cnt = calloc( n + 1, sizeof( spm_int_t ) );
    for ( spm_int_t j = 0; j < n; j++ ) {
        for ( spm_int_t e = spm->colptr[j] - b; e < spm->colptr[j + 1] - b; e++ ) {
            spm_int_t i = spm->rowptr[e] - b;
            cnt[j + 1]++;
            if ( i != j ) cnt[i + 1]++;
        }
    }
    for ( spm_int_t j = 0; j < n; j++ ) cnt[j + 1] += cnt[j];
    spm_int_t *rows = malloc( ( cnt[n] ? cnt[n] : 1 ) * sizeof( spm_int_t ) );
    spm_int_t *pos  = malloc( ( n ? n : 1 ) * sizeof( spm_int_t ) );
    memcpy( pos, cnt, n * sizeof( spm_int_t ) );
    for ( spm_int_t j = 0; j < n; j++ ) {
        for ( spm_int_t e = spm->colptr[j] - b; e < spm->colptr[j + 1] - b; e++ ) {
            spm_int_t i = spm->rowptr[e] - b;
            rows[pos[j]++] = i;
            if ( i != j ) rows[pos[i]++] = j;
        }
    }
    spm_int_t *ncol = malloc( ( n + 1 ) * sizeof( spm_int_t ) );
    spm_int_t  w    = 0;
    ncol[0] = 0;
    for ( spm_int_t j = 0; j < n; j++ ) {
        spm_int_t s = cnt[j], t = cnt[j + 1];
        qsort( rows + s, t - s, sizeof( spm_int_t ), cmp_int );
        for ( spm_int_t e = s; e < t; e++ ) {
            if ( e == s || rows[e] != rows[e - 1] ) rows[w++] = rows[e];
        }
        ncol[j + 1] = w;
    }
    spm_int_t added = w - spm->nnz;
    for ( spm_int_t j = 0; j <= n; j++ ) ncol[j] += b;
    for ( spm_int_t e = 0; e < w; e++ ) rows[e] += b;
    free( spm->colptr );
    free( spm->rowptr );
    spm->colptr = ncol;
    spm->rowptr = realloc( rows, ( w ? w : 1 ) * sizeof( spm_int_t ) );
    spm->nnz    = w;
    free( cnt );
    free( pos );
    spmUpdateComputedFields( spm );
    return added;
}

void spmUpdateComputedFields( spmatrix_t *spm )
{
    spm->gN   = spm->n;
    spm->gnnz = spm->nnz;
    if ( spm->dof > 0 ) {
        spm->nexp   = spm->n * spm->dof;
        spm->nnzexp = spm->nnz * spm->dof * spm->dof;
    }
    else {
        spm->nexp   = spm->dofs[spm->n] - spm->dofs[0];
        spm->nnzexp = value_count( spm );
    }
    spm->gNexp   = spm->nexp;
    spm->gnnzexp = spm->nnzexp;
}

double spmNorm( spm_normtype_t ntype, const spmatrix_t *spm )
{
    if ( ntype != SpmFrobeniusNorm || spm->values == NULL ||
         ( spm->flttype != SpmDouble && spm->flttype != SpmFloat ) || spm->dof < 1 ) {
        return -1.0;
    }
    const spm_int_t b = spm->baseval, d = spm->dof;
    double sum = 0.0;
    for ( spm_int_t j = 0; j < spm->n; j++ ) {
        for ( spm_int_t e = spm->colptr[j] - b; e < spm->colptr[j + 1] - b; e++ ) {
            spm_int_t i    = spm->rowptr[e] - b;
            double    mult = ( spm->mtxtype != SpmGeneral && i != j ) ? 2.0 : 1.0;
            for ( spm_int_t k = 0; k < d * d; k++ ) {
                double v = ( spm->flttype == SpmDouble ) ? ( (const double *)spm->values )[e * d * d + k]
                                                         : ( (const float *)spm->values )[e * d * d + k];
                sum += mult * v * v;
            }
        }
    }
    return sqrt( sum );
}

int spmExpand( const spmatrix_t *in, spmatrix_t *out )
{
    (void)in;
    (void)out;
    return SPM_ERR_NOTIMPLEMENTED;
}

int spmScatter( spmatrix_t *s, int root, const spmatrix_t *g, spm_int_t n, const spm_int_t *l2g, int bycol, SPM_Comm comm )
{
    (void)s; (void)root; (void)g; (void)n; (void)l2g; (void)bycol; (void)comm;
    return SPM_ERR_NOTIMPLEMENTED;
}

int spmGather( const spmatrix_t *s, int root, spmatrix_t *g )
{
    (void)s; (void)root; (void)g;
    return SPM_ERR_NOTIMPLEMENTED;
}

int spmLoad( spmatrix_t *spm, const char *filename )
{
    (void)spm; (void)filename;
    return SPM_ERR_NOTIMPLEMENTED;
}

int spmSave( const spmatrix_t *spm, const char *filename )
{
    (void)spm; (void)filename;
    return SPM_ERR_NOTIMPLEMENTED;
}

spm_int_t *spm_get_glob2loc( spmatrix_t *spm ) { return spm->glob2loc; }
