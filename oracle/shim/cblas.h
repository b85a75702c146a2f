/*
 * Empty stand-in for <cblas.h>.  The reference's common.h
 * (param_code/code_fft_1core/include/common.h:31) includes it but calls
 * nothing from it.  Test infrastructure only.
 */
#ifndef ORACLE_SHIM_CBLAS_H
#define ORACLE_SHIM_CBLAS_H
#endif
