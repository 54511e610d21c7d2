// Index checks of the checked build.
//
// Compiled with -DTC_BOUNDS_CHECK=1 (libthesiscode_b200_checked.so, built by
// `python -m thesiscode_b200.build --checked`), the hot-path kernels check
// every global-memory index against the extent of the array it addresses.
// Those kernels are the pair kernels (single and batched), source packing,
// the velocity and RK4 stage epilogues, the visiting-order keys, and the
// adjoint's row pass and its combination. The extent is the size of the allocation the library made, or
// the size the caller declared for its own array.
//
// An index outside [0, extent) is not accessed: a load gives zero and a store
// is skipped. The first such index is recorded in a per-device record that
// the host reads with tc_bounds_status. So a planning error (a wrong chunk
// count, offset or range) shows up as a record rather than as a memory fault.
// This build stands in for compute-sanitizer, which cannot be run here.
// Shared-memory indices are not checked: they come from compile-time tile
// shapes.
//
// In the release build TC_BC is the constant `true` and every check compiles
// away.
#pragma once
#include <cuda_runtime.h>

#ifndef TC_BOUNDS_CHECK
#define TC_BOUNDS_CHECK 0
#endif

namespace tcb {

// Violations since the last reset, then site, index and extent of the first.
struct BoundsRec {
  unsigned long long count;
  long long site, index, extent;
};

// Site ids (the header's TC_BC_* values).
enum BoundsSite : int {
  BC_PAIR_X = 1,     // pair kernels: target positions (points)
  BC_PAIR_PERM,      // pair kernels: target visiting order
  BC_PAIR_SRC,       // pair kernels: packed sources
  BC_PAIR_OUT,       // pair kernels: partial-sum stores (doubles)
  BC_BATCH_SEG,      // batched pair kernels: segment table
  BC_PACK_IN,        // packing: positions, vorticity, area (points)
  BC_PACK_OUT,       // packing: packed sources
  BC_EPI_PERM,       // velocity epilogue: visiting order
  BC_EPI_X,          // velocity epilogue: target positions (points)
  BC_EPI_PARTIAL,    // velocity epilogue: partial sums (doubles)
  BC_EPI_OUT,        // velocity epilogue: dX / dVort stores (points)
  BC_STAGE_PERM,     // stage epilogue: visiting orders
  BC_STAGE_STATE,    // stage epilogue: state and stage arrays of the row's class (points)
  BC_STAGE_PARTIAL,  // stage epilogue: partial sums (doubles)
  BC_STAGE_CHUNKS,   // stage epilogue: per-row chunk counts (batched runs)
  BC_STAGE_ACTIVE,   // stage epilogue: active-only arrays (vorticity, area, KE, sources)
  BC_STAGE_KEBLOCK,  // stage epilogue: per-block KE sums
  BC_ADJ_ROW_IN,     // adjoint row pass: per-panel inputs (ra, rb, rc)
  BC_ADJ_ROW_OUT,    // adjoint row pass: partial-sum stores (doubles)
  BC_ADJ_COMBINE,    // adjoint row combination: partial-sum reads (doubles)
  BC_ORDER_X,        // visiting-order keys: per-target inputs (positions, instance ids)
  BC_ORDER_KEYS,     // visiting-order keys: key and index stores
  BC_BATCH_KE,       // batched runs: per-instance KE sums' reads (KE, areas)
  BC_SITE_END
};

#if TC_BOUNDS_CHECK
__device__ __forceinline__ bool bounds_ok(BoundsRec* rec, int site, long long i, long long n) {
  if (i >= 0 && i < n) return true;
  if (rec && atomicAdd(&rec->count, 1ull) == 0ull) {
    rec->site = site;
    rec->index = i;
    rec->extent = n;
  }
  return false;
}
#define TC_BC(rec, site, i, n) (::tcb::bounds_ok((rec), (site), (long long)(i), (long long)(n)))
#else
#define TC_BC(rec, site, i, n) true
#endif

}  // namespace tcb
