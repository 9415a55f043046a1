/*
 * pastix/config.h -- configuration of the oracle build of the reference
 * (the header PaStiX's CMake generates from include/pastix/config.h.in).
 * TEST INFRASTRUCTURE ONLY.  One process (no MPI), no hwloc, no StarPU /
 * PaRSEC / CUDA, no Scotch / Metis (orderings are given by the caller),
 * 64-bit integers, OpenBLAS for CBLAS / LAPACKE.
 */
#ifndef _pastix_config_h_
#define _pastix_config_h_

#define PASTIX_VERSION_MAJOR 6
#define PASTIX_VERSION_MINOR 4
#define PASTIX_VERSION_MICRO 0

#define HAVE_SCHED_SETAFFINITY
#define HAVE_CLOCK_GETTIME
#define HAVE_ATOMIC_GCC_32_BUILTINS
#define HAVE_ATOMIC_GCC_64_BUILTINS
#define HAVE_STDARG_H
#define HAVE_UNISTD_H
#define HAVE_VA_COPY
#define HAVE_GETOPT_LONG
#define HAVE_GETRUSAGE
#define HAVE_GETOPT_H
#define HAVE_ERRNO_H
#define HAVE_STDDEF_H
#define HAVE_LIMITS_H
#define HAVE_STRING_H
#define HAVE_COMPLEX_H
#define HAVE_FALLTHROUGH
#define HAVE_BUILTIN_EXPECT
#define HAVE_GETLINE
#define HAVE_MKDTEMP

#define HAVE_OPENBLAS_SET_NUM_THREADS
void openblas_set_num_threads( int num_threads );
int  openblas_get_num_threads( void );

#define PASTIX_ARCH_X86
#define PASTIX_ARCH_X86_64

#define PASTIX_INT64

#if defined(HAVE_FALLTHROUGH)
#define pastix_attr_fallthrough __attribute__((fallthrough))
#else
#define pastix_attr_fallthrough do {} while(0)
#endif

#undef BEGIN_C_DECLS
#undef END_C_DECLS
#if defined(c_plusplus) || defined(__cplusplus)
# define BEGIN_C_DECLS extern "C" {
# define END_C_DECLS }
#else
#define BEGIN_C_DECLS          /* empty */
#define END_C_DECLS            /* empty */
#endif

#endif /* _pastix_config_h_ */
