// Internal interface of the segmented radix sort (k_sort.cu) for the other
// operator files.
#pragma once

#include "yq_keys.cuh"

namespace yq {

// One key of a (possibly multi-key) sort.
struct KeyJob {
  yq_column key;
  int desc, nulls_first;
  uint32_t* lossy = nullptr;  // set to non-zero when a key value would not round-trip its key words
};

// Words of the order-preserving key the sort builds for column `c` at most
// (text keys use fewer when their slots end in zero words); -1 = unsupported.
int sort_key_words_max(const yq_column& c);

// Segmented stable sort of `rows` rows by `jobs` (most significant first) into
// `out_perm`. With `keys_out` (single key only) the last pass also writes the
// transformed key words of the sorted rows ([rows][*kw_out] words; *kw_out = 0
// when every key is equal). With `defer_err` the call does not wait for the
// device to report errors: *err_out points at the workspace's error word.
//
// Leading key words that every row shares (found from the digit histogram:
// one bucket, the same in every segment) take no part in the passes: the
// passes, and `keys_out`, carry only the words below them. With `high_out`
// (8 words) the call reports the words it left out, least significant first:
// high_out[i] is key word *kw_out + i, in key form (after the DESC inversion).
int sort_segments_impl(const KeyJob* jobs, int njobs, uint32_t rows, const uint32_t* seg_offsets_host, int nseg,
                       uint32_t* out_perm, const yq_sort_config* cfg, void* workspace, size_t workspace_bytes,
                       cudaStream_t s, size_t* size_only, uint32_t* keys_out = nullptr, int* kw_out = nullptr,
                       bool defer_err = false, uint32_t** err_out = nullptr, uint32_t* high_out = nullptr);

// out[c][i] = in[c][perm[i]] for every column (yq_gather); with `only_if`,
// column c moves only when only_if[c] is null or *only_if[c] != 0 on the device.
int gather_impl(const yq_column* in, int32_t ncols, const uint32_t* perm, uint32_t rows, const yq_column* out,
                const uint32_t* const* only_if, cudaStream_t s);

}  // namespace yq
