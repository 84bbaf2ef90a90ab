// Types shared by the kernels and the grouped CP-stream engine: the
// arguments of one MTTKRP launch, the deterministic variant's long-chain
// workspace, and the items the grouped (many sessions per launch) entry
// points read out of a device table.
#pragma once

#include "alto_internal.cuh"

namespace alto {

struct FactorSet {
  const void* f[ALTO_MAX_MODES];
};

struct MttkrpArgs {
  const void* line;  // line records (LineRec16 / LineRec32)
  // DETERMINISTIC: per lane-group sub-range, its first and last run (slots
  // 2s and 2s+1: output row and R partial sums)
  uint32_t* det_rows;
  float* det_vals;
  const uint32_t* tile_iv;
  uint32_t nnz;
  uint32_t tile_nnz;
  uint32_t ntiles;
  int target;
  int stage_rows;  // rows of the shared staging buffer (0: never stage)
  // walks updating the output with atomics: consecutive tiles per block
  // chunk, the open run of each lane group carried from tile to tile
  uint32_t chunk_tiles;
  LineDecode dec;
  FactorSet fac;
  float* out;
};

// Workspace of the long chains (device): counters, then the chains
// {first slot, end slot, first segment, segments}, then the segments
// {chain, index in chain}, then each segment's R partial sums.
struct DetLong {
  uint32_t* counters;  // [0] long chains, [1] segments, [2] blocks of det_fix_final done
  uint4* chains;
  uint2* segs;
  float* segpart;
};

// A table of items of type T in device memory, `stride` bytes apart (for
// example one field of an array of per-session descriptors); the number of
// live items is read from *count when a kernel runs.
template <typename T>
struct Strided {
  const char* base;
  size_t stride;
  const int* count;
  __device__ __forceinline__ const T& operator[](int s) const {
    return *reinterpret_cast<const T*>(base + (size_t)s * stride);
  }
};

// One session's deterministic MTTKRP of one mode, ready to launch alone or
// in a group: kernel arguments, long-chain workspace, slot count, the
// record format of the line walked and the output's size (zeroed first).
// In a group, an item whose *active is 0 is skipped (active NULL: always).
struct DetItem {
  MttkrpArgs a;
  DetLong dl;
  uint32_t nslots;
  int hw;
  uint64_t out_floats;
  const int* active;
};

// Fill `item` for the deterministic MTTKRP of `mode` into `out` (building
// the mode's row-sorted copy and sizing the slot buffers as needed).
alto_status det_prepare(alto_tensor* t, int mode, const void* const* factors, int rank, float* out, DetItem* item,
                        cudaStream_t st);

// The deterministic MTTKRPs of a table of items at once; tile_off (device,
// [count + 1]) holds the prefix sums of the items' tile counts.  Every item
// has rank `rank`, record format `hw` and `nmodes` modes.  Each live item's
// output is zeroed and then gets exactly the sums, in the same order, that
// a launch of that item alone gives.  Fixed grids, everything read on the
// device: capturable once and relaunched with other items.
alto_status det_group_launch(Strided<DetItem> items, const uint32_t* tile_off, int rank, int hw, int nmodes,
                             cudaStream_t st);

// ---------------------------------------------------------- dense items

// W = (prod_{m in mask} grams[m] + shift I)^{-1} (solve_setup) for one session.
struct SetupItem {
  const double* grams;
  unsigned mask;
  int nmodes;
  int kind;
  double ridge;
  double* W;
  int* status;
  double* rho;
  const int* active;
};

// One session's G = U^T U, C = P^T U and change statistics
// (gram_cross_stats): nb blocks of rpb rows, partial sums in part.
struct GramItem {
  const float* P;
  const float* U;
  uint64_t I;
  uint64_t rpb;
  uint32_t nb;
  double* G;
  double* C;
  double* stats3;
  double* part;
  const int* active;
};

// Blocks and rows per block gram_cross_stats uses for I rows (so a grouped
// pass splits each session exactly as its own call does).
void gram_split(uint64_t I, uint32_t* nb, uint64_t* rpb);

// Grouped solve set-up (one CTA per item, R <= 64).
alto_status setup_group_launch(Strided<SetupItem> items, int max_items, int R, cudaStream_t st);
// Grouped gram_cross_stats: block_off (device, [count + 1]) holds the prefix
// sums of the items' nb; red_off likewise for their reduction blocks.
alto_status gram_group_ready(int R);  // before capturing gram_group_launch at rank R
alto_status gram_group_launch(Strided<GramItem> items, const uint32_t* block_off, const uint32_t* red_off,
                              int max_items, int R, cudaStream_t st);
// Reduction blocks of one GramItem's pass at rank R.
uint32_t gram_reduce_blocks(int R);

}  // namespace alto

// ------------------------------------------------ stream groups
//
// A stream group runs the inner iterations of several CP-stream sessions
// (same rank, mode count, stream mode and line record formats) in the same
// launches: one CUDA graph, captured when the group is made, loops over
// steps (one inner iteration of every member still running) and reads the
// members' descriptors from a device table, so it is relaunched unchanged
// however the membership changes.  A session alone runs in a group of one.

namespace alto {

struct StreamGroup;

// Whether the session's batches can run in a group (the CP-stream model at
// rank 8, 16 or 32 with 3 to 5 modes, once it has a batch).
bool stream_groupable(const alto_stream_session* s);
// After the batch is prepared: the per-mode MTTKRP items and the buffer
// sizes the group's kernels use; the batch's iteration state cleared.
alto_status group_prepare_session(alto_stream_session* s);
bool group_fits(const StreamGroup* g, const alto_stream_session* s);
// A group of up to `capacity` members like `like`, working on stream st.
alto_status group_create(const alto_stream_session* like, int capacity, cudaStream_t st, StreamGroup** out);
void group_destroy(StreamGroup* g);
// The members of the next launches (each prepared and fitting the group).
alto_status group_set(StreamGroup* g, alto_stream_session* const* members, int k);
// Up to max_steps inner iterations of every member, one graph launch.
alto_status group_launch(StreamGroup* g, int max_steps);
// After the group's stream is drained: per member whether it runs on, its
// inner iterations, stop flag and failed-Cholesky info (any may be NULL).
alto_status group_states(StreamGroup* g, int* running, int* done, int* stop, int* info);

}  // namespace alto

namespace alto {
// The serving loop's steps of one batch: prepare it (everything before the
// inner iterations; *grouped tells whether it then runs in a group, else
// stream_run_ungrouped runs its iterations and finish); after its group
// has run it to the end, finish it (forgetting, prev <- current, time rows).
alto_status stream_prepare_grouped(alto_stream_session* s, const alto_coo* b, const double* init_vals,
                                   uint64_t n_init, bool* grouped);
alto_status stream_run_ungrouped(alto_stream_session* s, int* inner);
alto_status stream_finish_grouped(alto_stream_session* s, int* inner);
bool stream_group_key_equal(const alto_stream_session* a, const alto_stream_session* b);
void stream_set_cuda_stream(alto_stream_session* s, cudaStream_t st);
}  // namespace alto
