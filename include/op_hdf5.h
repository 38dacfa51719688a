/*
 * op_hdf5.h -- OP2's HDF5 mesh I/O (op2/include/op_hdf5.h, implemented in
 * op2/src/externlib/op_hdf5.cpp:66-1121 over the HDF5 library).  libop2b reads
 * and writes the HDF5 file format itself (no HDF5 library needed): files
 * written by HDF5 libraries with their default settings are read -- groups as
 * symbol tables or compact link lists, contiguous, compact or chunked
 * datasets (deflate, shuffle, fletcher32), numbers of either byte order,
 * fixed-length strings -- and files are written in the layout those libraries
 * write by default (superblock version 0, symbol-table groups, contiguous
 * little-endian datasets).
 *
 * File layout, as the reference's: a set is a one-element int dataset named
 * after the set; a map is a [from size][dim] dataset with int attributes
 * "size" and "dim" and a string attribute "type"; a dat a [set size][dim]
 * dataset with "size" (bytes per element), "dim" and "type"; a constant a
 * [dim] dataset with "dim" and "type".  Names may be paths ("/a/b/c"); the
 * groups on them are created when writing.
 *
 * Where the reference prints a message and exits the program, these
 * functions record the message (op2b_last_error) and return NULL or leave
 * the file as it was.
 */
#ifndef OP2B_OP_HDF5_H
#define OP2B_OP_HDF5_H

#include "op2b.h"

#ifdef __cplusplus
extern "C" {
#endif

/* op_hdf5.cpp:66-90: a set of the size the one-element dataset `name` holds */
op_set op_decl_set_hdf5(char const *file, char const *name);
/* op_hdf5.cpp:92-138: a set of the first extent of `set_dataset_name` */
op_set op_decl_set_hdf5_infer_size(char const *file, char const *name,
                                   char const *set_dataset_name);
/* op_hdf5.cpp:144-233: the map in dataset `name` (int or 64-bit integers
 * within int range); its extents must be [from size][dim].  NULL with a
 * message when the file has no such dataset. */
op_map op_decl_map_hdf5(op_set from, op_set to, int dim, char const *file,
                        char const *name);
/* op_hdf5.cpp:239-338: the dat in dataset `name`, converted to `type` when
 * the file holds another number type; its extents must be [set size][dim] */
op_dat op_decl_dat_hdf5(op_set set, int dim, char const *type, char const *file,
                        char const *name);
/* op_hdf5.cpp:617-698: `dim` values of dataset `name` into const_data, as
 * `type`; the dataset's "dim" attribute must equal dim */
void op_get_const_hdf5(char const *name, int dim, char const *type,
                       char *const_data, char const *file_name);
/* op_hdf5.cpp:344-611: every set, map and dat declared so far, as the
 * library holds them now (current values, current numbering), into a new
 * file */
void op_dump_to_hdf5(char const *file_name);
/* op_hdf5.cpp:704-805: constant `name` added to file_name (created if
 * missing); a dataset of that name already there is an error */
void op_write_const_hdf5(char const *name, int dim, char const *type,
                         char *const_data, char const *file_name);
/* op_hdf5.cpp:882-1121: the dat's current values, in the order the
 * application declared them, into dataset dat->name (or path_name) of
 * file_name: an existing dataset is overwritten after its size, dim and type
 * attributes are checked, else a new one is made; the file is created if
 * missing */
void op_fetch_data_hdf5_file(op_dat dat, char const *file_name);
void op_fetch_data_hdf5_file_path(op_dat dat, char const *file_name,
                                  char const *path_name);

/* ---- op2b extensions: the file format from the host, without op_init or a
 * GPU.  Types are OP2 names ("int", "long", "long long", "float", "double",
 * and their equivalents).  Return 0, or -1 with a message. */

/* rank, extents and OP2 type name ("string" for strings, "UNRECOGNISED"
 * for other types) of dataset `path`; 1 when there is none */
int op2b_h5_info(const char *file, const char *path, int *rank, long long dims[8],
                 char *type, int type_len);
/* all `count` elements of dataset `path`, converted to `type` */
int op2b_h5_read(const char *file, const char *path, const char *type, void *out,
                 long long count);
/* a dataset at `path` (replacing one there, making the groups on the way) in
 * `file` (created if missing) */
int op2b_h5_write(const char *file, const char *path, const char *type, int rank,
                  const long long *dims, const void *data);
/* attribute `name` of the object at `path`: `count` numbers of `type`, or,
 * with type "string", the string `data` in `count` bytes (0: its length) */
int op2b_h5_set_attr(const char *file, const char *path, const char *name,
                     const char *type, int count, const void *data);
/* attribute `name` as text (a string, or numbers separated by spaces); 1 when
 * there is none */
int op2b_h5_get_attr(const char *file, const char *path, const char *name, char *out,
                     int out_len);
/* every object of the file, one a line ("/a/" a group, "/a/b" a dataset);
 * returns the bytes the list needs with its terminating zero */
long long op2b_h5_list(const char *file, char *out, long long out_len);

#ifdef __cplusplus
}
#endif

#endif /* OP2B_OP_HDF5_H */
