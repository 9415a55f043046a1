/* spm/src/common.h -- SpM's internal header, included by bcsc/bvec_zlapmr.c
 * for its distributed helpers; one process needs none of them.
 * TEST INFRASTRUCTURE ONLY. */
#ifndef ORACLE_SPM_SRC_COMMON_H
#define ORACLE_SPM_SRC_COMMON_H
#include "spm.h"
#endif
