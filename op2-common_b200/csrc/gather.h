// Inverse maps and the owner-computes ("gather") indirect loops.  Internal.
#pragma once

#include "loops.h"
#include "op2b.h"

namespace op2b {

// Inverse of a map from -> to: for target t, entries off[t] .. off[t+1]-1 of
// ent hold element*dim + slot of every (element, slot) mapping to t, sorted
// ascending.  rows lists the targets with at least one entry (all targets
// when all_rows).
struct InvMap {
  const long long *off;
  const int *ent;
  const int *rows;
  int nrows, nto, dim;
  bool all_rows;
};

const InvMap *get_inverse_map(op_map map);
void release_inverse_maps();  // also drops the slot records built on them

// Four slots per cell for res_calc's 4-lanes-per-cell gather: other cell,
// the edge's nodes, role (bit 30 of n2) and valid (bit 31 of n2).  usable is
// false when some cell has more than four incident edges.
struct SlotRecords {
  const int *o, *n1;
  const unsigned *n2;
  int ncell;
  bool usable;
  // Corner form (built on request by get_corner_records): in a quadrilateral
  // mesh the <= 4 interior edges of a cell touch at most four distinct nodes.
  // cn[c] lists them (first appearance over slots 0..3, an edge's first node
  // before its second; unused corners repeat the first one) and byte s of
  // meta[c] describes slot s: bit 0 valid, bit 1 role (the cell is the edge's
  // second cell), bits 2-3 / 4-5 the corners of the edge's first / second
  // node.  corners is false when some cell's edges touch more than four nodes.
  const int *cn;
  const unsigned *meta;
  bool corners;
  // Flux-ring form (built on request by build_ring_records, for the fused
  // res_calc + bres_calc and res_calc over corner records): cells are split
  // into ring_ctas contiguous ranges of ring_span cells, one per CTA, swept in
  // tiles of ring_nt cells.  16 bits per slot in ring[c] (slots 0-1 in .x,
  // 2-3 in .y, low half first): bits 14-15 clear = the cell computes the
  // edge's flux (its other cell comes later in the range) and puts it at
  // entry (bits 0-11) of the CTA's shared-memory ring; bit 15 = the flux was
  // put there by the other cell, earlier in the range; bit 14 = the other cell
  // lies outside the range: the cell computes the flux for itself alone
  // (kept in its tile's scratch, not the ring).
  const uint2 *ring;
  int ring_ctas, ring_span, ring_nt;
};
// entries of a CTA's flux ring (a power of two: the 12-bit index of ring[])
#define OP2B_RING_ENTRIES 4096
const SlotRecords *get_slot_records(op_map pecell, op_map pedge);
const SlotRecords *get_corner_records(op_map pecell, op_map pedge);
void release_slot_records();

template <typename T>
cudaError_t launch_res_calc_gather4(const LaunchCtx &c, const SlotRecords &s, const T *x,
                                    const T *q, const T *adt, T *res, const AirConst<T> &k);
template <typename T>
cudaError_t launch_res_calc_gather_cell4(const LaunchCtx &c, const SlotRecords &s, const T *x,
                                         const T *q, const T *adt, T *res,
                                         const AirConst<T> &k);
// airfoil_pipe.cu: slot records, operands staged in shared memory by cp.async
// one cell ahead (block = threads per CTA: 64, 96, 128 or 256)
template <typename T>
cudaError_t launch_res_calc_gather_pipe(const LaunchCtx &c, const SlotRecords &s, const T *x,
                                        const T *q, const T *adt, T *res, const AirConst<T> &k,
                                        int block);
// airfoil_pipe.cu: slot records, operands of the next cell prefetched into
// registers while the current one is computed (persistent grid)
template <typename T>
cudaError_t launch_res_calc_gather_regpipe(const LaunchCtx &c, const SlotRecords &s, const T *x,
                                           const T *q, const T *adt, T *res,
                                           const AirConst<T> &k, int block);

// Build the flux-ring records for nctas ranges and tiles of nt cells; false
// (the corner kernels then serve) when the corner records are missing, two
// cells share more than one edge, or some flux would have to wait in the
// ring longer than OP2B_RING_ENTRIES allows (cells' neighbours too far apart
// in the numbering: renumbering the mesh brings them close).  Cached.
bool build_ring_records(const SlotRecords *s, int nctas, int nt);

// which gather kernel res_calc uses (option "gather_kernel")
#define OP2B_GATHER_CSR 1    // one thread per cell walking the inverse map
#define OP2B_GATHER_LANES 2  // four threads per cell, shuffled together
#define OP2B_GATHER_CELL4 3  // one thread per cell, four slot records, unrolled
#define OP2B_GATHER_PIPE 4   // cell4's order, shared-memory software pipeline
#define OP2B_GATHER_REGPIPE 5  // cell4's order, register software pipeline
#define OP2B_GATHER_CORNER 6   // the register pipeline over corner records
#define OP2B_GATHER_RING 7     // corner records, each in-range flux computed once (flux ring)

// airfoil_pipe.cu: the register pipeline over corner records (four node
// gathers per cell instead of eight); block 64, 128 or 256 threads, minb the
// __launch_bounds__ minimum CTAs per SM (1 = no register cap)
template <typename T>
cudaError_t launch_res_calc_gather_corner(const LaunchCtx &c, const SlotRecords &s, const T *x,
                                          const T *q, const T *adt, T *res,
                                          const AirConst<T> &k, int block, int minb);

// Boundary records for bres_calc's gather, one per (cell, boundary edge) in
// ascending (cell, edge) order: {cell, node 1, node 2, edge}; a record that
// continues the previous record's cell stores -1 - cell there.  Built from
// the maps (immutable between renumberings) and cached like the slot records.
struct BresRecords {
  const int4 *rec;
  int n;
};
const BresRecords *get_bres_records(op_map pbecell, op_map pbedge);
template <typename T>
cudaError_t launch_bres_calc_records(const LaunchCtx &c, const BresRecords &b, const int *bound,
                                     const T *x, const T *q, const T *adt, T *res,
                                     const AirConst<T> &k);

// Link the boundary edges into the corner records for the fused res_calc +
// bres_calc: a boundary cell's boundary edges go into the unused slots of its
// corner record, after its interior slots and in edge order (meta bit 6, the
// edge's nodes as corners, o = the boundary edge).  False when some boundary
// edge finds no unused slot or has a node that is not a corner of its cell, or
// the corner records are not usable; the loops then run one after the other.
bool link_boundary_records(const SlotRecords *s, const BresRecords *b, op_map pbecell);
// airfoil_pipe.cu: the fused kernel (block 128 or 256).  zero_res: res is
// known to be all zeros (the update before left it so without writing it):
// the kernel starts each cell's sums from 0 instead of reading res.
template <typename T>
cudaError_t launch_res_bres_corner(const LaunchCtx &c, const SlotRecords &s,
                                   const BresRecords &b, const int *bound, const T *x,
                                   const T *q, const T *adt, T *res, const AirConst<T> &k,
                                   int block, bool zero_res = false);
// airfoil_ring.cu: res_calc (bound = nullptr) or the fused res_calc +
// bres_calc over the flux-ring records (s.ring set; one CTA per range)
template <typename T>
cudaError_t launch_res_ring(const LaunchCtx &c, const SlotRecords &s, const int *bound,
                            const T *x, const T *q, const T *adt, T *res, const AirConst<T> &k,
                            bool zero_res);

template <typename T>
cudaError_t launch_res_calc_gather(const LaunchCtx &c, const InvMap &inv, const int *pedge,
                                   const int *pecell, const T *x, const T *q, const T *adt,
                                   T *res, const AirConst<T> &k);
template <typename T>
cudaError_t launch_bres_calc_gather(const LaunchCtx &c, const InvMap &inv, const int *pbedge,
                                    const int *bound, const T *x, const T *q, const T *adt,
                                    T *res, const AirConst<T> &k);

}  // namespace op2b
