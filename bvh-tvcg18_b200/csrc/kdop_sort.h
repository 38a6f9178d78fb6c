// kdop_sort.h -- device radix sort and exclusive scan (kdop_sort.cu).
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace kdop {

// Words of scratch radix_sort_pairs needs for n keys.
size_t radix_scratch_words(int64_t n);
// Stable ascending sort of (keys, vals), n < 2^32; keys_tmp / vals_tmp hold n
// each; scratch radix_scratch_words(n) words (8-byte aligned).  Reads the
// keys' common bits back to the host once (synchronises the stream).
cudaError_t radix_sort_pairs(uint64_t* keys, uint32_t* vals, uint64_t* keys_tmp, uint32_t* vals_tmp, int64_t n,
                             uint32_t* scratch, cudaStream_t st);
// Words of scratch exclusive_scan_u32 needs for n counts.
size_t scan_scratch_words(int64_t n);
// out[i] = in[0] + ... + in[i-1] (in == out allowed).
cudaError_t exclusive_scan_u32(const uint32_t* in, uint32_t* out, int64_t n, uint32_t* scratch, cudaStream_t st);

}  // namespace kdop

struct kdop_scene;
namespace kdop {
// Sorts the last traversal's n candidate rows by (pair, tet of A, tet of B)
// and, after kdop_contacts, regroups the n_contacts contact rows and the
// records in that order.  work: sort_results_bytes(n, n_contacts) bytes.
cudaError_t sort_results(kdop_scene* s, int64_t n, int64_t n_contacts, void* work, cudaStream_t st);
size_t sort_results_bytes(int64_t n, int64_t n_contacts);
}  // namespace kdop
