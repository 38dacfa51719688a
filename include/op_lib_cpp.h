/*
 * op_lib_cpp.h -- the OP2 C++ convenience layer over libop2b's C ABI.
 *
 * Replaces op2/include/op_lib_cpp.h:57-203 for applications built against
 * libop2b: run-time type checks (type_error), op_decl_dat<T>,
 * op_decl_const2<T>, op_arg_gbl<T>, op_arg_info<T>, op_opt_arg_gbl<T>,
 * op_decl_dat_temp<T>, op_fetch_data<T>, op_fetch_data_idx<T>.
 *
 * op_decl_const(dim, type, &var) -- which the reference's sequential header
 * turns into a type check only, leaving kernels to read the global -- is a
 * macro here that records the constant under the variable's own name, because
 * device loops receive constants by name (e.g. "gam", "qinf").
 */
#ifndef OP2B_OP_LIB_CPP_H
#define OP2B_OP_LIB_CPP_H

/* the standard headers an application gets through the reference's
 * op_lib_core.h:43-68 */
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <strings.h>

#include <cstddef>
#include <iostream>
#include <limits>
#include <stdexcept>
#include <utility>

#include "op2b.h"
#include "op2b_plan.h"
#include "op_hdf5.h"

/* op2/include/op_lib_core.h:246-249 */
#ifndef MIN
#define MIN(a, b) ((a < b) ? (a) : (b))
#endif
#ifndef MAX
#define MAX(a, b) ((a > b) ? (a) : (b))
#endif

typedef unsigned int uint;
typedef long long ll;
typedef unsigned long long ull;

inline int type_error(const double *, const char *type) {
  return strcmp(type, "double") && strcmp(type, "double:soa");
}
inline int type_error(const float *, const char *type) {
  return strcmp(type, "float") && strcmp(type, "float:soa");
}
inline int type_error(const int *, const char *type) {
  return strcmp(type, "int") && strcmp(type, "int:soa");
}
inline int type_error(const uint *, const char *type) {
  return strcmp(type, "uint") && strcmp(type, "uint:soa");
}
inline int type_error(const ll *, const char *type) {
  return strcmp(type, "ll") && strcmp(type, "ll:soa");
}
inline int type_error(const ull *, const char *type) {
  return strcmp(type, "ull") && strcmp(type, "ull:soa");
}
inline int type_error(const bool *, const char *type) {
  return strcmp(type, "bool") && strcmp(type, "bool:soa");
}

/* print-and-exit on a failed call, as the reference does (op_lib_core.cpp:393-395) */
inline void op2b_check_handle(const void *h, const char *what) {
  if (!h) {
    printf("%s error -- %s\n", what, op2b_last_error());
    exit(-1);
  }
}

template <class T>
op_dat op_decl_dat(op_set set, int dim, char const *type, T *data, char const *name) {
  if (type_error(data, type)) {
    printf("incorrect type specified for dataset \"%s\" \n", name);
    exit(1);
  }
  op_dat d = op_decl_dat_char(set, dim, type, sizeof(T), (char *)data, name);
  op2b_check_handle(d, "op_decl_dat");
  return d;
}

template <class T>
op_dat op_decl_dat_temp(op_set set, int dim, char const *type, T *, char const *name) {
  op_dat d = op_decl_dat_temp_char(set, dim, type, sizeof(T), name);
  op2b_check_handle(d, "op_decl_dat_temp");
  return d;
}

inline int op_free_dat_temp(op_dat dat) { return op_free_dat_temp_char(dat); }

template <class T> void op_decl_const2(char const *name, int dim, char const *type, T *data) {
  if (type_error(data, type)) {
    printf("incorrect type specified for constant \"%s\" \n", name);
    exit(1);
  }
  op_decl_const_char(dim, type, sizeof(T), (char *)data, name);
}

template <class T>
void op2b_decl_const_named(int dim, char const *type, T *data, char const *name) {
  op_decl_const2(name, dim, type, data);
}
#define op_decl_const(dim, type, dat) op2b_decl_const_named(dim, type, dat, #dat)

template <class T> op_arg op_arg_gbl(T *data, int dim, char const *type, op_access acc) {
  return op_arg_gbl_char((char *)data, dim, type_error(data, type) ? "error" : type, sizeof(T),
                         acc);
}

template <class T> op_arg op_arg_info(T *data, int dim, char const *type, int ref) {
  return op_arg_info_char((char *)data, dim, type_error(data, type) ? "error" : type, sizeof(T),
                          ref);
}

template <class T>
op_arg op_opt_arg_gbl(int opt, T *data, int dim, char const *type, op_access acc) {
  return op_opt_arg_gbl_char(opt, (char *)data, dim, type_error(data, type) ? "error" : type,
                             sizeof(T), acc);
}

template <class T> void op_fetch_data(op_dat dat, T *usr_ptr) {
  op_fetch_data_char(dat, (char *)usr_ptr);
}

template <class T> void op_fetch_data_idx(op_dat dat, T *usr_ptr, int low, int high) {
  op_fetch_data_idx_char(dat, (char *)usr_ptr, low, high);
}

#endif /* OP2B_OP_LIB_CPP_H */
