/*
 * op2b.h -- C ABI of libop2b, a single-GPU (B200, sm_100a) backend behind the
 * OP2 C API.  Every entry point here uses plain C types, pointers and sizes.
 *
 * Each declaration names the reference interface it replaces
 * (OP2-Common, paths relative to the OP2-Common tree).  Types and constants
 * keep the reference's names and values so that OP2 application code compiles
 * unchanged against include/op_seq.h (which includes this file).
 *
 * Execution model: all op_dat storage lives in device memory (AoS, one
 * element = dim contiguous values).  op_decl_* copy user arrays in; op_fetch_*
 * copy results out; op_par_loop runs a hand-written CUDA kernel chosen by the
 * loop's name and checked against its argument signature.  There is no CPU
 * fallback: a loop without a device implementation is an error.
 *
 * Errors: functions returning int return 0 on success and a negative code
 * otherwise; op2b_last_error() gives the message.  Functions whose reference
 * signature returns a handle return NULL on error.
 */
#ifndef OP2B_H
#define OP2B_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Access modes and argument kinds: op2/include/op_lib_core.h:108-119 */
#define OP_READ 0
#define OP_WRITE 1
#define OP_RW 2
#define OP_INC 3
#define OP_MIN 4
#define OP_MAX 5
#define OP_WORK 6

#define OP_ARG_GBL 0
#define OP_ARG_DAT 1
#define OP_ARG_IDX 2
#define OP_ARG_INFO 3

/* Plan staging modes: op2/include/op_lib_core.h:121-125 */
#define OP_STAGE_NONE 0
#define OP_STAGE_INC 1
#define OP_STAGE_ALL 2
#define OP_STAGE_PERMUTE 3
#define OP_COLOR2 4

typedef int op_access;
typedef int op_arg_type;

/* op_set_core: op2/include/op_lib_core.h:134-145 (same leading fields) */
typedef struct op_set_core {
  int index;
  int size;
  char const *name;
  int core_size;
  int exec_size;
  int nonexec_size;
} op_set_core;
typedef op_set_core *op_set;

/* op_map_core: op2/include/op_lib_core.h:149-160.  `map` is the library's
 * host copy (AoS [from->size][dim]); map_d the device copy. */
typedef struct op_map_core {
  int index;
  op_set from, to;
  int dim;
  int *map;
  int *map_d;
  char const *name;
} op_map_core;
typedef op_map_core *op_map;

/* op_dat_core: op2/include/op_lib_core.h:164-179.  data_d is the device
 * array.  `data` is a host copy of the values as declared (zeros for a NULL
 * source), as the reference's op_decl_dat keeps one, in the current
 * numbering (op_renumber reorders it with the device copy); loops run on the
 * device and leave it as it was -- op_fetch_data returns current values.
 * With the option host_mirror = 0 it is NULL. */
typedef struct op_dat_core {
  int index;
  op_set set;
  int dim, size; /* size = bytes per element (dim * sizeof(type)) */
  char *data, *data_d;
  char const *type, *name;
} op_dat_core;
typedef op_dat_core *op_dat;

/* op_arg: op2/include/op_lib_core.h:183-199 (same fields) */
typedef struct op_arg {
  int index;
  op_dat dat;
  op_map map;
  int dim, idx, size;
  char *data, *data_d;
  int *map_data, *map_data_d;
  char const *type;
  op_access acc;
  op_arg_type argtype;
  int sent;
  int opt;
} op_arg;

#define OP_ID ((op_map)NULL)  /* op2/include/op_lib_c.h:47 */
#define OP_GBL ((op_map)NULL) /* op2/include/op_lib_c.h:48 */

/* ---- initialisation: op2/include/op_lib_c.h:75-76, op_lib_core.cpp:287-389
 * argv tokens OP_BLOCK_SIZE=, OP_PART_SIZE=, OP_CACHE_LINE_SIZE= are parsed as
 * in op_set_args (op2/src/core/op_lib_core.cpp:205-281). */
void op_init(int argc, char **argv, int diags);
void op_exit(void); /* op_lib_c.h:111, frees every handle and device array */

/* ---- declarations: op2/include/op_lib_c.h:78-92 */
op_set op_decl_set(int size, char const *name);
op_map op_decl_map(op_set from, op_set to, int dim, int *imap, char const *name);
op_dat op_decl_dat_char(op_set set, int dim, char const *type, int type_size,
                        char *data, char const *name);
/* op_decl_dat_temp_char fails (NULL) if a dat of the same set, dim, type and
 * name exists (op_lib_core.cpp:638-651); op_free_dat_temp_char returns 1
 * when it freed the dat, -1 otherwise (:653-680). */
op_dat op_decl_dat_temp_char(op_set set, int dim, char const *type,
                             int type_size, char const *name);
int op_free_dat_temp_char(op_dat dat);
/* op_lib_c.h:85-86, op_lib_core.cpp:581-636: a dat on `set` sharing the
 * storage of `dat` (or of the dat declared from the array `dat`), host copy
 * and device array; `set` may not be larger than the dat's set.  op_renumber
 * refuses to run while overlays exist. */
op_dat op_decl_dat_overlay(op_set set, op_dat dat);
op_dat op_decl_dat_overlay_ptr(op_set set, char *dat);
void op_decl_const_char(int dim, char const *type, int type_size, char *dat,
                        char const *name);

/* ---- loop arguments: op2/include/op_lib_c.h:94-102, op_lib_core.cpp:831-1061 */
op_arg op_arg_dat(op_dat dat, int idx, op_map map, int dim, char const *type,
                  op_access acc);
op_arg op_opt_arg_dat(int opt, op_dat dat, int idx, op_map map, int dim,
                      char const *type, op_access acc);
op_arg op_arg_gbl_char(char *data, int dim, const char *type, int type_size,
                       op_access acc);
op_arg op_opt_arg_gbl_char(int opt, char *data, int dim, const char *type,
                           int type_size, op_access acc);
op_arg op_arg_info_char(char *data, int dim, const char *type, int type_size,
                        int ref);
op_arg op_arg_idx(int idx, op_map map);

/* ---- parallel loops.  The generic entry point takes the argument list as
 * an array (the op_par_loop of op2/include/op_seq.h, without the host kernel
 * pointer); the named entry points have the signature of the reference
 * translator's host stubs (translator-v2/resources/templates/cpp/
 * loop_host.hpp.jinja:35-41), e.g. op_par_loop_res_calc(name, set, 8 args). */
int op_par_loop_c(char const *name, op_set set, int nargs, op_arg *args);

void op_par_loop_save_soln(char const *name, op_set set, op_arg a0, op_arg a1);
void op_par_loop_adt_calc(char const *name, op_set set, op_arg a0, op_arg a1,
                          op_arg a2, op_arg a3, op_arg a4, op_arg a5);
void op_par_loop_res_calc(char const *name, op_set set, op_arg a0, op_arg a1,
                          op_arg a2, op_arg a3, op_arg a4, op_arg a5,
                          op_arg a6, op_arg a7);
void op_par_loop_bres_calc(char const *name, op_set set, op_arg a0, op_arg a1,
                           op_arg a2, op_arg a3, op_arg a4, op_arg a5);
void op_par_loop_update(char const *name, op_set set, op_arg a0, op_arg a1,
                        op_arg a2, op_arg a3, op_arg a4, op_arg a5, op_arg a6,
                        op_arg a7);

/* ---- data out: op2/include/op_lib_c.h:104-121, op_lib_core.cpp:1283-1370 */
void op_fetch_data_char(op_dat dat, char *usr_ptr);
void op_fetch_data_idx_char(op_dat dat, char *usr_ptr, int low, int high);
void op_print_dat_to_binfile(op_dat dat, const char *file_name);
void op_print_dat_to_txtfile(op_dat dat, const char *file_name);

/* ---- sizes, timers, diagnostics: op_lib_c.h:113-117, op_lib_core.h:305-337 */
int op_get_size(op_set set);
void op_timers(double *cpu, double *et);
void op_timing_output(void);
void op_diagnostic_output(void);
void op_rank(int *rank);
/* partitioning (op_lib_core.h:395-402): one rank owns every set, so these
 * do nothing, as in the reference's single-node builds
 * (op_dummy_singlenode.cpp:144-200); op_is_root returns 1. */
void op_partition(const char *lib_name, const char *lib_routine, op_set prime_set,
                  op_map prime_map, op_dat coords);
void op_partition_ptr(const char *lib_name, const char *lib_routine, op_set prime_set,
                      int *prime_map, double *coords);
void op_partition_reverse(void);
void op_partition_destroy(void);
int op_is_root(void);
/* op_printf (op_lib_core.h:289) and the allocation wrappers (op_lib_core.h:
 * 423-429): host memory, 64-byte aligned, for application code. */
void op_printf(const char *format, ...);
void *op_malloc(size_t size);
void *op_calloc(size_t num, size_t size);
void *op_realloc(void *ptr, size_t size);
void op_free(void *ptr);

/* ---- renumbering: op_renumber / op_renumber_ptr of
 * op2/src/externlib/op_renumber.cpp:224-516 (declared for MPI builds in the
 * reference).  The base map's target set is ordered by a GPU reverse
 * Cuthill-McKee (the reference uses PT-Scotch's Gibbs-Poole-Stockmeyer), the
 * order is propagated to every set reachable through declared maps, and maps
 * and dats are reordered on the device.  Plans built before are dropped.
 * op_fetch_data_idx keeps returning data in the original numbering. */
void op_renumber(op_map base);
void op_renumber_ptr(int *ptr);

/* ---- op2b extensions (no reference counterpart unless stated) ---------- */

/* op_renumber returning a status; stats (may be NULL) receives the base
 * map's bandwidth {max, average} before and after, as the reference prints
 * (op_renumber.cpp:489-502). */
int op2b_renumber(op_map base, long stats[4]);
/* perm[i] = current index of the element declared as i (identity if the set
 * was never renumbered; returns 1 then, 0 otherwise, -1 on error). */
int op2b_set_permutation(op_set set, int *perm);

/* Message of the last failed call on this thread ("" if none). */
const char *op2b_last_error(void);
/* 0 when op_init has run and the CUDA device answered. */
int op2b_status(void);

/* Upload host data into an existing dat (op_upload_dat of
 * op2/include/op_lib_core.h:349 with the data supplied by the caller). */
int op2b_dat_upload(op_dat dat, const char *src, size_t bytes);
/* Device pointer of a dat / map (for interop; plain device addresses).  Any
 * deferred loop is launched first, and the runtime no longer computes ahead
 * (speculate_adt) into a dat whose pointer was handed out. */
void *op2b_dat_device_ptr(op_dat dat);
void *op2b_map_device_ptr(op_map map);

/* Indirect-increment strategy for res_calc/bres_calc style loops
 * (replaces the choice between the reference's atomics and colouring
 * templates, translator-v2/.../cuda/loop_host.hpp.jinja:143-173,341-389):
 *   0 = segmented atomics, 1 = block + thread colouring over the plan,
 *   2 = plan staging with atomics only on cells shared between blocks. */
#define OP2B_INC_ATOMIC 0
#define OP2B_INC_COLOR 1
#define OP2B_INC_HYBRID 2
/* 3 = owner computes: each target element sums its increments, in element
 * order, through the map's inverse (no atomics, no colours; bit-exact with
 * the reference's sequential loop on the same numbering). */
#define OP2B_INC_GATHER 3
int op2b_set_option(const char *key, long value);

/* Kernel sources for loops that have no hand-written device kernel.  The
 * reference's code generator compiles each user kernel into a device loop
 * before the application is built (translator-v2); libop2b compiles it at
 * the loop's first call instead, for sm_100a with NVRTC, from the source
 * registered here under the loop's name, or else from the file <name>.h on
 * OP2B_KERNEL_PATH (default: the working directory), the reference's
 * one-kernel-per-header convention.  Preludes (helper functions, types; or
 * user_types.h where it exists) are placed before every kernel.  Direct
 * arguments in every access mode, indirect OP_READ and OP_INC, op_arg_idx and
 * op_arg_gbl OP_READ/OP_INC/OP_MIN/OP_MAX are supported; anything else is an
 * error.  A NULL source forgets the name's registration.  Registering drops
 * the compiled modules.  Return 0, -1 on error. */
int op2b_register_kernel(const char *name, const char *source);
int op2b_register_prelude(const char *source);
long op2b_get_option(const char *key);

/* Per-loop device time (CUDA events on the library stream), launches and
 * algorithmic bytes moved per call, as accumulated since op_init or the last
 * reset; name = loop name.  Returns -1 if the loop never ran. */
int op2b_loop_stats(const char *name, double *total_ms, long *calls,
                    double *bytes_per_call, double *last_ms);
void op2b_reset_stats(void);
/* Number of kernels the library launched since op_init. */
long op2b_kernel_launches(void);

/* Stream the library launches on (cudaStream_t as void*); NULL = the
 * library's own non-blocking stream. */
int op2b_set_stream(void *stream);
void *op2b_get_stream(void);
/* Block until every launched kernel has finished; returns a CUDA error code. */
int op2b_synchronize(void);

/* Halo exchange of a partitioned mesh, device side (replaces the packing of
 * op_exchange_halo, op2/src/mpi/op_mpi_rt_support.cpp:61-200, and its CUDA
 * gather/scatter kernels, op2/src/mpi/op_mpi_cuda_kernels.cu:44-136).
 * op2b_dat_pack: buf (device) receives rows rows[0..n) of dat, one row of
 * dat->size bytes after the other.  op2b_dat_unpack: rows rows[0..n) of dat
 * (or, rows NULL, the contiguous rows first .. first+n-1) receive the
 * buffer's rows.  Asynchronous on the library's stream; 0 or -1. */
int op2b_dat_pack(op_dat dat, const int *rows, int n, void *buf);
int op2b_dat_unpack(op_dat dat, const int *rows, int first, int n, const void *buf);

/* The update loop (q = qold - res/adt, res = 0, rms += sum of del^2, maxerr
 * and errloc from the largest del^2) for callers that cannot allocate device
 * memory: an application whose device memory is all held by its own pool, or
 * a latency-critical path that must not pay the device-wide synchronisation
 * of cudaMalloc/cudaFree.  It allocates nothing: the reduction scratch is a
 * fixed array inside the library (about 512 KiB held on every GPU that loads
 * the library, until exit).  No counterpart in the reference.
 *   qold, q, res (4 doubles per cell), adt (1 per cell): the caller's device
 *   arrays; rms, maxerr, errloc: the caller's device scalars, updated as
 *   op_arg_gbl OP_INC / OP_MAX / op_arg_info do (rms += ..., maxerr and
 *   errloc replaced only when beaten).  Results are in device memory when the
 *   work on `stream` (a cudaStream_t; NULL = legacy default stream) is done.
 *   ncell must not exceed 4,194,304; larger values return -1 with a message.
 *   qold, q and res must be 16-byte aligned, adt, rms and maxerr 8-byte,
 *   errloc 4-byte (cudaMalloc'd arrays are); a misaligned pointer returns -1
 *   with a message before anything is launched.
 *   The first call on a device (and the first after the device was reset)
 *   looks up the scratch array's device address; make that call before any
 *   stream capture.  Calls share the one
 *   scratch array, so calls whose work can overlap on the GPU race: serialise
 *   them.  Works without op_init (the device current on the calling thread is
 *   used). */
int op2b_update_noalloc(int ncell, const double *qold, double *q, double *res,
                        const double *adt, double *rms, double *maxerr, int *errloc,
                        void *stream);

#ifdef __cplusplus
}
#endif

#endif /* OP2B_H */
