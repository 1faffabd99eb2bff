/* Declarations only (see cblas.h in this folder). */
#ifndef REFSHIM_LAPACKE_H_
#define REFSHIM_LAPACKE_H_
typedef int lapack_int;
#ifdef __cplusplus
extern "C" {
#endif
void dpotrf_(char*, lapack_int*, double*, lapack_int*, lapack_int*);
void dpotrs_(char*, lapack_int*, lapack_int*, double*, lapack_int*, double*, lapack_int*, lapack_int*);
void dgelsy_(lapack_int*, lapack_int*, lapack_int*, double*, lapack_int*, double*, lapack_int*,
             lapack_int*, double*, lapack_int*, double*, lapack_int*, lapack_int*);
#ifdef __cplusplus
}
#endif
#endif
