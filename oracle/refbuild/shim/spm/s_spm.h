/* s_spm.h -- the one SpM dense helper the reference's solve step names
 * (a debug print of a right-hand side).  TEST INFRASTRUCTURE ONLY. */
#ifndef ORACLE_s_SPM_H
#define ORACLE_s_SPM_H
#include "spm.h"
static inline void s_spmDensePrint( FILE *f, spm_int_t m, spm_int_t n, const void *A, spm_int_t lda )
{
    const float *a = (const float *)A;
    for ( spm_int_t j = 0; j < n; j++ )
        for ( spm_int_t i = 0; i < m; i++ )
            fprintf( f, "%ld %ld %e\n", (long)i, (long)j, creal( (spm_complex64_t)a[j * lda + i] ) );
}
#endif
