// The stream slicer on the device: the reference's StreamingSparseTensor
// (src/streaming_sptensor.cpp:69-327) over a whole COO tensor resident in HBM.
//
//   construction (:69-125)  one stable LSD radix sort of a packed key whose
//                           fields are the modes in the order (t, t+1, ...)
//                           mod N, the stream mode most significant: the
//                           order tt_sort produces (src/sort.cpp:477-519);
//                           then the first-seen relabel of every other mode.
//   next_dynamic_batch      batch cuts on the host from two small tables
//   (:196-264)              built once: the first sorted position of every
//                           time step, and per mode the number of distinct
//                           indices seen before it.  A batch is a view of the
//                           resident arrays; one kernel writes its local
//                           time indices.
//   stream_prev (:284-327)  the same view over the last `previous` steps.
//
// The first-seen relabel needs no second pass over the nonzeros before the
// relabel itself: for every index value the smallest sorted position
// holding it (an atomic minimum, one per run of equal values in a warp),
// then a sort of the (mode, first position) -> value pairs -- as many as
// the modes' lengths, not the nonzeros -- which lists each mode's values in
// first-appearance order: label = rank in that list.  Since labels follow
// first appearance, the running maximum the reference keeps in _prev_dim is
// the number of distinct indices before the batch end, a binary search of
// the batch end in the sorted first positions.
#include <algorithm>
#include <cstring>
#include <new>

#include "alto_internal.cuh"

namespace alto {

alto_status check_coo_shape(const alto_coo* coo);

namespace {

constexpr uint32_t kNone = 0xffffffffu;

// Bit fields of the sort key: mode m at bits [shift[m], shift[m] + bits[m]).
struct SortFields {
  int nmodes;
  int shift[ALTO_MAX_MODES];
  int bits[ALTO_MAX_MODES];
  uint64_t dims[ALTO_MAX_MODES];
  uint64_t first_off[ALTO_MAX_MODES];  // offset of mode m's first-seen table
};

struct InPtrs {
  const void* cidx[ALTO_MAX_MODES];
};

__device__ __forceinline__ void put_field(uint64_t x, int shift, int bits, uint64_t& lo, uint64_t& hi) {
  if (!bits) return;  // (a one-row mode: x is 0, and shift may be 128)
  if (shift < 64) {
    lo |= x << shift;
    if (shift && shift + bits > 64) hi |= x >> (64 - shift);
  } else {
    hi |= x << (shift - 64);
  }
}

__device__ __forceinline__ uint32_t get_field(uint64_t lo, uint64_t hi, int shift, int bits) {
  if (!bits) return 0;
  uint64_t v;
  if (shift < 64) {
    v = lo >> shift;
    if (shift && shift + bits > 64) v |= hi << (64 - shift);
  } else {
    v = hi >> (shift - 64);
  }
  return (uint32_t)(v & ((1ull << bits) - 1));
}

// Sort keys and the identity payload; an index outside its mode sets *err
// (and is clamped to 0, so nothing downstream leaves its table).
template <int IB>
__global__ void slice_key_kernel(InPtrs in, SortFields f, uint32_t nnz, uint64_t* __restrict__ klo,
                                 uint64_t* __restrict__ khi, uint32_t* __restrict__ perm, int* __restrict__ err) {
  for (uint64_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nnz; i += gridDim.x * blockDim.x) {
    uint64_t lo = 0, hi = 0;
    for (int m = 0; m < f.nmodes; ++m) {
      uint64_t x = IB == 8 ? ((const uint64_t*)in.cidx[m])[i] : (uint64_t)((const uint32_t*)in.cidx[m])[i];
      if (x >= f.dims[m]) {
        atomicOr(err, 1);
        x = 0;
      }
      put_field(x, f.shift[m], f.bits[m], lo, hi);
    }
    klo[i] = lo;
    if (khi) khi[i] = hi;
    perm[i] = (uint32_t)i;
  }
}

// Sorted order: the stream mode's time step, the original index of every
// other mode (relabelled in place later), the values gathered, and per
// index value its first sorted position (lowest lane of each run of equal
// values in a warp takes the atomic minimum).
template <typename VT>
__global__ void slice_decode_kernel(const uint64_t* __restrict__ klo, const uint64_t* __restrict__ khi,
                                    const uint32_t* __restrict__ perm, SortFields f, int t, uint32_t nnz,
                                    const VT* __restrict__ vin, VT* __restrict__ vout, uint32_t* __restrict__ gtime,
                                    uint32_t* __restrict__ idx, uint32_t* __restrict__ first) {
  const uint64_t stride = gridDim.x * blockDim.x;
  const int lane = threadIdx.x & 31;
  for (uint64_t base = blockIdx.x * blockDim.x; base < nnz; base += stride) {
    const uint64_t i = base + threadIdx.x;
    const bool valid = i < nnz;
    const unsigned vmask = __ballot_sync(0xffffffffu, valid);
    if (!valid) continue;
    const uint64_t lo = klo[i], hi = khi ? khi[i] : 0;
    vout[i] = vin[perm[i]];
    for (int m = 0; m < f.nmodes; ++m) {
      const uint32_t v = get_field(lo, hi, f.shift[m], f.bits[m]);
      if (m == t) {
        gtime[i] = v;
        continue;
      }
      idx[(size_t)m * nnz + i] = v;
      const unsigned peers = __match_any_sync(vmask, v);
      if (lane == __ffs(peers) - 1) atomicMin(first + f.first_off[m] + v, (uint32_t)i);
    }
  }
}

// The first-seen relabel.  first[] holds, for every value of every
// non-stream mode (mode m at first_off[m]), the first sorted position that
// holds it (kNone if none does).  Sorting the pairs (mode, first position)
// -> value puts each mode's values in first-appearance order, which is the
// label order: no pass over the nonzeros beyond the final relabel.
__device__ __forceinline__ int mode_of(const SortFields& f, int t, uint64_t q) {
  int m = 0;
  for (int k = 0; k < f.nmodes; ++k)
    if (k != t && q >= f.first_off[k] && q < f.first_off[k] + f.dims[k]) m = k;
  return m;
}

__global__ void slice_first_pairs_kernel(const uint32_t* __restrict__ first, SortFields f, int t, uint64_t nfirst,
                                         uint64_t* __restrict__ key, uint32_t* __restrict__ val) {
  for (uint64_t q = blockIdx.x * blockDim.x + threadIdx.x; q < nfirst; q += gridDim.x * blockDim.x) {
    const int m = mode_of(f, t, q);
    key[q] = ((uint64_t)m << 32) | first[q];
    val[q] = (uint32_t)(q - f.first_off[m]);
  }
}

// From the sorted pairs: the r-th value of mode m to appear gets label r;
// label[m][value] = r (in first[]'s storage) and iperm[m][r] = value (the
// reference's Permutation iperms).
__global__ void slice_label_table_kernel(const uint64_t* __restrict__ skey, const uint32_t* __restrict__ sval,
                                         SortFields f, uint64_t nfirst, uint32_t* __restrict__ label,
                                         uint32_t* __restrict__ iperm) {
  for (uint64_t q = blockIdx.x * blockDim.x + threadIdx.x; q < nfirst; q += gridDim.x * blockDim.x) {
    const uint64_t k = skey[q];
    if ((uint32_t)k == kNone) continue;
    const int m = (int)(k >> 32);
    const uint32_t r = (uint32_t)(q - f.first_off[m]);
    label[f.first_off[m] + sval[q]] = r;
    iperm[f.first_off[m] + r] = sval[q];
  }
}

// idx[m][p] = the label of its original index.
__global__ void slice_relabel_kernel(uint32_t* __restrict__ idx, const uint32_t* __restrict__ label,
                                     SortFields f, int t, uint32_t nnz) {
  const int m = blockIdx.y;
  if (m == t) return;
  uint32_t* ix = idx + (size_t)m * nnz;
  const uint32_t* lb = label + f.first_off[m];
  for (uint64_t p = blockIdx.x * blockDim.x + threadIdx.x; p < nnz; p += gridDim.x * blockDim.x)
    ix[p] = lb[ix[p]];
}

// off[b] = first sorted position with time >= b (b = 0..T).  Position p
// owns the steps (time[p-1], time[p]] (p = nnz owns the steps after the
// last time).
__global__ void slice_steps_kernel(const uint32_t* __restrict__ gtime, uint32_t nnz, uint32_t T,
                                   uint32_t* __restrict__ off) {
  for (uint64_t p = blockIdx.x * blockDim.x + threadIdx.x; p <= nnz; p += gridDim.x * blockDim.x) {
    const uint64_t lo = p == 0 ? 0 : (uint64_t)gtime[p - 1] + 1;
    const uint64_t hi = p == nnz ? T : gtime[p];
    for (uint64_t b = lo; b <= hi; ++b) off[b] = p;
  }
}

// cnt[m][b] = distinct indices of mode m before off[b]: the values of m
// first seen before it, a binary search in m's sorted first positions.
__global__ void slice_counts_kernel(const uint64_t* __restrict__ skey, SortFields f, int t, uint32_t T,
                                    const uint32_t* __restrict__ off, uint32_t* __restrict__ cnt) {
  const uint64_t n = (uint64_t)f.nmodes * (T + 1);
  for (uint64_t q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
    const int m = (int)(q / (T + 1));
    const uint32_t b = (uint32_t)(q % (T + 1));
    if (m == t) {
      cnt[q] = 0;
      continue;
    }
    const uint64_t target = ((uint64_t)m << 32) | off[b];
    uint64_t lo = f.first_off[m], hi = lo + f.dims[m];
    while (lo < hi) {
      const uint64_t mid = (lo + hi) / 2;
      if (skey[mid] < target)
        lo = mid + 1;
      else
        hi = mid;
    }
    cnt[q] = (uint32_t)(lo - f.first_off[m]);
  }
}

// out[i] = time[begin + i] - first_step, i < n.
__global__ void slice_local_time_kernel(const uint32_t* __restrict__ gtime, uint32_t begin, uint32_t n,
                                        uint32_t first_step, uint32_t* __restrict__ out) {
  for (uint64_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    out[i] = gtime[begin + i] - first_step;
}

unsigned grid_n(uint64_t n, int threads) {
  uint64_t b = (n + threads - 1) / threads;
  if (b > 148ull * 32) b = 148ull * 32;
  return (unsigned)(b ? b : 1);
}

size_t align256(size_t x) { return (x + 255) / 256 * 256; }

}  // namespace
}  // namespace alto

using namespace alto;

struct alto_slicer {
  int N = 0, t = 0;
  uint64_t nnz = 0, T = 0;
  uint64_t dims[ALTO_MAX_MODES] = {};
  alto_dtype vdt = ALTO_F64;
  cudaStream_t st = nullptr;
  // (from the library's pool, on st; alto_slicer_destroy waits for the
  // whole device before they return to it, as cudaFree would)
  PoolBuf idx;    // [N][nnz] uint32: labels; the stream mode's row holds batch-local time
  PoolBuf gtime;  // [nnz] uint32: time step of each sorted position
  PoolBuf vals;   // [nnz] values in sorted order, input dtype
  PoolBuf ptime;  // stream_prev's time indices
  PoolBuf iperm;  // per non-stream mode, original index of each label
  uint64_t iperm_off[ALTO_MAX_MODES] = {};
  std::vector<uint32_t> off;  // [T + 1]
  std::vector<uint32_t> cnt;  // [N][T + 1]
  uint64_t ptr = 0, step = 0;  // _nnz_ptr, _batch_num
  uint64_t prev_dim[ALTO_MAX_MODES] = {};
  uint64_t bdims[ALTO_MAX_MODES] = {}, pdims[ALTO_MAX_MODES] = {};
  const void* bptr[ALTO_MAX_MODES] = {};
  const void* pptr[ALTO_MAX_MODES] = {};
  std::vector<uint64_t> cut_start, cut_end, cut_dims;  // alto_slicer_cut_all's batches
  PoolBuf steptab;                                    // each time step's batch first step
  uint64_t tdims[ALTO_MAX_MODES] = {};  // the whole tensor's view
  const void* tptr[ALTO_MAX_MODES] = {};
};

namespace {

alto_status slicer_build(alto_slicer* s, const alto_coo* coo) {
  const int N = s->N, t = s->t;
  const uint64_t nnz = s->nnz;
  const uint32_t n32 = (uint32_t)nnz;
  cudaStream_t st = s->st;

  // key fields: the last mode of the cyclic order is least significant
  SortFields f{};
  f.nmodes = N;
  int total = 0;
  for (int k = N - 1; k >= 0; --k) {
    const int m = (t + k) % N;
    f.bits[m] = s->dims[m] <= 1 ? 0 : 64 - __builtin_clzll(s->dims[m] - 1);
    f.shift[m] = total;
    f.dims[m] = s->dims[m];
    total += f.bits[m];
  }
  if (total > 128) {
    set_error("slicer key needs %d bits (at most 128)", total);
    return ALTO_ERR_UNSUPPORTED;
  }
  uint64_t nfirst = 0;
  for (int m = 0; m < N; ++m) {
    f.first_off[m] = nfirst;
    if (m != t) nfirst += s->dims[m];
  }
  for (int m = 0; m < N; ++m) s->iperm_off[m] = f.first_off[m];

  const bool two_words = total > 64;
  const int vbytes = coo->val_dtype == ALTO_F64 ? 8 : 4;
  const size_t cap = std::max<uint64_t>(nnz, 1);
  // the sort buffers serve the nonzeros' sort, then the relabel's pair sort
  const size_t scap = std::max<uint64_t>(cap, nfirst);
  ALTO_TRY(s->idx.ensure((size_t)N * cap * 4, st));
  ALTO_TRY(s->gtime.ensure(cap * 4, st));
  ALTO_TRY(s->vals.ensure(cap * vbytes, st));
  ALTO_TRY(s->iperm.ensure(std::max<uint64_t>(nfirst, 1) * 4, st));

  PoolBuf scratch;  // (transient: the library pool keeps it for the next slicer)
  size_t o = 0;
  const size_t o_lo0 = o; o = align256(o + scap * 8);
  const size_t o_lo1 = o; o = align256(o + scap * 8);
  const size_t o_hi0 = o; o = align256(o + (two_words ? cap * 8 : 0));
  const size_t o_hi1 = o; o = align256(o + (two_words ? cap * 8 : 0));
  const size_t o_p0 = o; o = align256(o + scap * 4);
  const size_t o_p1 = o; o = align256(o + scap * 4);
  const size_t o_cnt = o; o = align256(o + radix_scratch_bytes(scap));
  const size_t o_first = o; o = align256(o + std::max<uint64_t>(nfirst, 1) * 4);
  const size_t o_step = o; o = align256(o + (size_t)(N + 1) * (s->T + 1) * 4);
  const size_t o_err = o; o = align256(o + 8);  // [0] index range, [1] sort look-back
  const size_t o_vin = o; o = align256(o + (coo->on_device ? 0 : cap * vbytes));
  const size_t o_cin = o; o = align256(o + (coo->on_device ? 0 : (size_t)N * cap * coo->index_bytes));
  ALTO_TRY(scratch.ensure(o, st));
  char* sb = scratch.as<char>();
  uint64_t* klo[2] = {(uint64_t*)(sb + o_lo0), (uint64_t*)(sb + o_lo1)};
  uint64_t* khi[2] = {two_words ? (uint64_t*)(sb + o_hi0) : nullptr, two_words ? (uint64_t*)(sb + o_hi1) : nullptr};
  uint32_t* pm[2] = {(uint32_t*)(sb + o_p0), (uint32_t*)(sb + o_p1)};
  uint32_t* first = (uint32_t*)(sb + o_first);
  uint32_t* d_off = (uint32_t*)(sb + o_step);
  uint32_t* d_cnt = d_off + (s->T + 1);
  int* d_err = (int*)(sb + o_err);

  InPtrs in{};
  const void* vin = coo->vals;
  if (coo->on_device) {
    for (int m = 0; m < N; ++m) in.cidx[m] = coo->cidx[m];
  } else if (nnz) {
    for (int m = 0; m < N; ++m) {
      char* dst = sb + o_cin + (size_t)m * cap * coo->index_bytes;
      ALTO_TRY_CUDA(cudaMemcpyAsync(dst, coo->cidx[m], nnz * coo->index_bytes, cudaMemcpyHostToDevice, st));
      in.cidx[m] = dst;
    }
    ALTO_TRY_CUDA(cudaMemcpyAsync(sb + o_vin, coo->vals, nnz * vbytes, cudaMemcpyHostToDevice, st));
    vin = sb + o_vin;
  }
  ALTO_TRY_CUDA(cudaMemsetAsync(d_err, 0, 8, st));
  ALTO_TRY_CUDA(cudaMemsetAsync(first, 0xff, std::max<uint64_t>(nfirst, 1) * 4, st));

  const dim3 gm(grid_n(nnz, 256), N);
  if (nnz) {
    if (coo->index_bytes == 8)
      slice_key_kernel<8><<<grid_n(nnz, 256), 256, 0, st>>>(in, f, n32, klo[0], khi[0], pm[0], d_err);
    else
      slice_key_kernel<4><<<grid_n(nnz, 256), 256, 0, st>>>(in, f, n32, klo[0], khi[0], pm[0], d_err);
    ALTO_LAUNCHED();
    int cur = 0;
    ALTO_TRY(radix_sort_pairs(klo, khi, pm, n32, total, sb + o_cnt, d_err + 1, st, &cur));
    if (coo->val_dtype == ALTO_F64)
      slice_decode_kernel<double><<<grid_n(nnz, 256), 256, 0, st>>>(
          klo[cur], khi[cur], pm[cur], f, t, n32, (const double*)vin, s->vals.as<double>(), s->gtime.as<uint32_t>(),
          s->idx.as<uint32_t>(), first);
    else
      slice_decode_kernel<float><<<grid_n(nnz, 256), 256, 0, st>>>(
          klo[cur], khi[cur], pm[cur], f, t, n32, (const float*)vin, s->vals.as<float>(), s->gtime.as<uint32_t>(),
          s->idx.as<uint32_t>(), first);
    ALTO_LAUNCHED();
  }
  // first-seen labels: the (mode, first position) -> value pairs sorted
  const uint64_t* skey = nullptr;  // the sorted pairs' keys
  if (nfirst) {
    slice_first_pairs_kernel<<<grid_n(nfirst, 256), 256, 0, st>>>(first, f, t, nfirst, klo[0], pm[0]);
    ALTO_LAUNCHED();
    uint64_t* nohi[2] = {nullptr, nullptr};
    int pc = 0;
    const int pair_bits = 32 + (N > 1 ? 32 - __builtin_clz((unsigned)(N - 1)) : 0);
    ALTO_TRY(radix_sort_pairs(klo, nohi, pm, (uint32_t)nfirst, pair_bits, sb + o_cnt, d_err + 1, st, &pc));
    slice_label_table_kernel<<<grid_n(nfirst, 256), 256, 0, st>>>(klo[pc], pm[pc], f, nfirst, first,
                                                                  s->iperm.as<uint32_t>());
    ALTO_LAUNCHED();
    if (nnz) {
      slice_relabel_kernel<<<gm, 256, 0, st>>>(s->idx.as<uint32_t>(), first, f, t, n32);
      ALTO_LAUNCHED();
    }
    skey = klo[pc];
  }
  slice_steps_kernel<<<grid_n(nnz + 1, 256), 256, 0, st>>>(s->gtime.as<uint32_t>(), n32, (uint32_t)s->T, d_off);
  ALTO_LAUNCHED();
  if (skey) {
    slice_counts_kernel<<<grid_n((uint64_t)N * (s->T + 1), 256), 256, 0, st>>>(skey, f, t, (uint32_t)s->T, d_off,
                                                                                 d_cnt);
    ALTO_LAUNCHED();
  } else {
    ALTO_TRY_CUDA(cudaMemsetAsync(d_cnt, 0, (size_t)N * (s->T + 1) * 4, st));
  }

  int err[2] = {0, 0};
  s->off.assign(s->T + 1, 0);
  s->cnt.assign((size_t)N * (s->T + 1), 0);
  ALTO_TRY_CUDA(cudaMemcpyAsync(s->off.data(), d_off, (s->T + 1) * 4, cudaMemcpyDeviceToHost, st));
  ALTO_TRY_CUDA(cudaMemcpyAsync(s->cnt.data(), d_cnt, (size_t)N * (s->T + 1) * 4, cudaMemcpyDeviceToHost, st));
  ALTO_TRY_CUDA(cudaMemcpyAsync(err, d_err, sizeof(err), cudaMemcpyDeviceToHost, st));
  ALTO_TRY_CUDA(cudaStreamSynchronize(st));  // (also: host COO outlives its copies; scratch is freed below)
  if (err[0]) {
    set_error("an index of the tensor is outside its mode's dims");
    return ALTO_ERR_INVALID;
  }
  if (err[1]) {
    set_error("the slicer's device sort gave up waiting on a preceding tile");
    return ALTO_ERR_TIMEOUT;
  }
  return ALTO_OK;
}

// A view over sorted positions [start, end) whose stream-mode row is `time`.
void fill_view(const alto_slicer* s, uint64_t start, uint64_t end, const uint64_t* dims, const void** ptrs,
               const uint32_t* time, alto_coo* out) {
  const int vb = s->vdt == ALTO_F64 ? 8 : 4;
  for (int m = 0; m < s->N; ++m)
    ptrs[m] = m == s->t ? (const void*)time : (const void*)(s->idx.as<uint32_t>() + (size_t)m * s->nnz + start);
  out->nmodes = s->N;
  out->dims = dims;
  out->nnz = end - start;
  out->cidx = ptrs;
  out->index_bytes = 4;
  out->vals = s->vals.as<char>() + start * vb;
  out->val_dtype = s->vdt;
  out->on_device = 1;
}

}  // namespace

extern "C" {

alto_status alto_slicer_create(const alto_coo* coo, int stream_mode, alto_cuda_stream stream, alto_slicer** out) {
  if (!out) {
    set_error("out is NULL");
    return ALTO_ERR_INVALID;
  }
  *out = nullptr;
  ALTO_TRY(check_coo_shape(coo));
  if (stream_mode < 0 || stream_mode >= coo->nmodes) {
    set_error("stream_mode %d outside 0..%d", stream_mode, coo->nmodes - 1);
    return ALTO_ERR_INVALID;
  }
  if ((uint64_t)coo->nmodes * (coo->nnz + 1) >= (1ull << 32)) {
    set_error("nmodes * (nnz + 1) must stay below 2^32 for the slicer");
    return ALTO_ERR_UNSUPPORTED;
  }
  alto_slicer* s = new (std::nothrow) alto_slicer();
  if (!s) {
    set_error("host allocation failed");
    return ALTO_ERR_NOMEM;
  }
  s->N = coo->nmodes;
  s->t = stream_mode;
  s->nnz = coo->nnz;
  for (int m = 0; m < s->N; ++m) s->dims[m] = coo->dims[m];
  s->T = s->dims[stream_mode];
  s->vdt = coo->val_dtype;
  s->st = (cudaStream_t)stream;
  alto_status r = slicer_build(s, coo);
  if (r != ALTO_OK) {
    delete s;
    return r;
  }
  *out = s;
  return ALTO_OK;
}

}  // extern "C"

namespace {

// One next_dynamic_batch cut (src/streaming_sptensor.cpp:196-264) on the
// host tables: advances the position and the step, sets s->bdims and
// s->prev_dim; [start, end) and the batch's first step are returned.
void cut_batch(alto_slicer* s, uint64_t nnz_threshold, uint64_t timeslice_limit, uint64_t* start_out,
               uint64_t* end_out, uint64_t* first_out) {
  const uint64_t first = s->step;
  const uint64_t start = std::max<uint64_t>(s->ptr, s->off[std::min(s->step, s->T)]);
  uint64_t end = start;
  while (end - start < nnz_threshold && end < s->nnz) {
    end = std::max<uint64_t>(end, s->off[std::min(s->step + 1, s->T)]);
    ++s->step;
    if (s->step - first >= timeslice_limit) break;
  }
  const uint64_t endstep = std::min(s->step, s->T);
  for (int m = 0; m < s->N; ++m) {
    if (m == s->t) {
      s->bdims[m] = s->step - first;
    } else {
      s->bdims[m] = std::max<uint64_t>(s->cnt[(size_t)m * (s->T + 1) + endstep], 1);
      s->prev_dim[m] = s->bdims[m];
    }
  }
  s->ptr = end;
  *start_out = start;
  *end_out = end;
  *first_out = first;
}

}  // namespace

namespace alto {
namespace {
// out[i] = time[begin + i] - first_of[time[begin + i]], i < n: every
// position's batch-local time, given each time step's batch first step.
__global__ void slice_local_time_all_kernel(const uint32_t* __restrict__ gtime, uint64_t begin, uint64_t n,
                                            const uint32_t* __restrict__ first_of, uint32_t* __restrict__ out) {
  for (uint64_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t tt = gtime[begin + i];
    out[begin + i] = tt - first_of[tt];
  }
}
}  // namespace
}  // namespace alto

extern "C" {

alto_status alto_slicer_next(alto_slicer* s, uint64_t nnz_threshold, uint64_t timeslice_limit, alto_coo* batch,
                             int* got) {
  if (!s || !batch || !got) {
    set_error("slicer, batch or got is NULL");
    return ALTO_ERR_INVALID;
  }
  *got = 0;
  if (s->ptr == s->nnz) return ALTO_OK;  // the reference returns NULL
  uint64_t start, end, first;
  cut_batch(s, nnz_threshold, timeslice_limit, &start, &end, &first);
  uint32_t* time = s->idx.as<uint32_t>() + (size_t)s->t * s->nnz + start;
  if (end > start) {
    slice_local_time_kernel<<<grid_n(end - start, 256), 256, 0, s->st>>>(
        s->gtime.as<uint32_t>(), (uint32_t)start, (uint32_t)(end - start), (uint32_t)first, time);
    ALTO_LAUNCHED();
  }
  fill_view(s, start, end, s->bdims, s->bptr, time, batch);
  *got = 1;
  return ALTO_OK;
}

alto_status alto_slicer_cut_all(alto_slicer* s, uint64_t nnz_threshold, uint64_t timeslice_limit,
                                uint64_t* nbatches) {
  if (!s || !nbatches) {
    set_error("slicer or nbatches is NULL");
    return ALTO_ERR_INVALID;
  }
  const int N = s->N;
  s->cut_start.clear();
  s->cut_end.clear();
  s->cut_dims.clear();
  const uint64_t p0 = s->ptr;
  std::vector<uint32_t> first_of(s->T + 1, 0);
  while (s->ptr < s->nnz) {
    uint64_t start, end, first;
    cut_batch(s, nnz_threshold, timeslice_limit, &start, &end, &first);
    for (uint64_t b = first; b < std::min(s->step, s->T); ++b) first_of[b] = (uint32_t)first;
    s->cut_start.push_back(start);
    s->cut_end.push_back(end);
    for (int m = 0; m < N; ++m) s->cut_dims.push_back(s->bdims[m]);
  }
  if (s->nnz > p0) {
    ALTO_TRY(s->steptab.ensure((s->T + 1) * 4, s->st));
    ALTO_TRY_CUDA(cudaMemcpyAsync(s->steptab.p, first_of.data(), (s->T + 1) * 4, cudaMemcpyHostToDevice, s->st));
    slice_local_time_all_kernel<<<grid_n(s->nnz - p0, 256), 256, 0, s->st>>>(
        s->gtime.as<uint32_t>(), p0, s->nnz - p0, s->steptab.as<uint32_t>(), s->idx.as<uint32_t>() + (size_t)s->t * s->nnz);
    ALTO_LAUNCHED();
  }
  *nbatches = s->cut_start.size();
  return ALTO_OK;
}

alto_status alto_slicer_batch(alto_slicer* s, uint64_t b, alto_coo* out) {
  if (!s || !out || b >= s->cut_start.size()) {
    set_error("bad slicer, batch number or out");
    return ALTO_ERR_INVALID;
  }
  const uint64_t start = s->cut_start[b];
  fill_view(s, start, s->cut_end[b], s->cut_dims.data() + b * s->N, s->bptr,
            s->idx.as<uint32_t>() + (size_t)s->t * s->nnz + start, out);
  return ALTO_OK;
}

alto_status alto_slicer_last_batch(const alto_slicer* s, int* last) {
  if (!s || !last) {
    set_error("slicer or last is NULL");
    return ALTO_ERR_INVALID;
  }
  *last = s->ptr == s->nnz;
  return ALTO_OK;
}

alto_status alto_slicer_stream_prev(alto_slicer* s, uint64_t previous, alto_coo* out, int* got) {
  if (!s || !out || !got) {
    set_error("slicer, out or got is NULL");
    return ALTO_ERR_INVALID;
  }
  *got = 0;
  if (s->step == 0) return ALTO_OK;  // the reference returns NULL
  const uint64_t start_time = previous < s->step ? s->step - previous : 0;
  const uint64_t start = s->off[std::min(start_time, s->T)], end = s->ptr;
  const uint64_t n = end > start ? end - start : 0;
  ALTO_TRY(s->ptime.ensure(std::max<uint64_t>(n, 1) * 4, s->st));
  if (n) {
    slice_local_time_kernel<<<grid_n(n, 256), 256, 0, s->st>>>(s->gtime.as<uint32_t>(), (uint32_t)start,
                                                                (uint32_t)n, (uint32_t)start_time,
                                                                s->ptime.as<uint32_t>());
    ALTO_LAUNCHED();
  }
  for (int m = 0; m < s->N; ++m) s->pdims[m] = m == s->t ? s->step - start_time : s->prev_dim[m];
  fill_view(s, start, start + n, s->pdims, s->pptr, s->ptime.as<uint32_t>(), out);
  *got = 1;
  return ALTO_OK;
}

alto_status alto_slicer_tensor(const alto_slicer* s, alto_coo* out) {
  if (!s || !out) {
    set_error("slicer or out is NULL");
    return ALTO_ERR_INVALID;
  }
  alto_slicer* w = const_cast<alto_slicer*>(s);
  for (int m = 0; m < s->N; ++m) w->tdims[m] = s->dims[m];
  fill_view(s, 0, s->nnz, w->tdims, w->tptr, s->gtime.as<uint32_t>(), out);
  return ALTO_OK;
}

alto_status alto_slicer_iperm(alto_slicer* s, int mode, uint64_t* host_out, uint64_t* count) {
  if (!s || !count || mode < 0 || mode >= s->N) {
    set_error("bad slicer, mode or count");
    return ALTO_ERR_INVALID;
  }
  const uint64_t n = mode == s->t ? s->dims[mode] : s->cnt[(size_t)mode * (s->T + 1) + s->T];
  *count = n;
  if (!host_out) return ALTO_OK;
  if (mode == s->t) {
    for (uint64_t i = 0; i < n; ++i) host_out[i] = i;
    return ALTO_OK;
  }
  std::vector<uint32_t> tmp(n);
  if (n)
    ALTO_TRY_CUDA(cudaMemcpyAsync(tmp.data(), s->iperm.as<uint32_t>() + s->iperm_off[mode], n * 4,
                                  cudaMemcpyDeviceToHost, s->st));
  ALTO_TRY_CUDA(cudaStreamSynchronize(s->st));
  for (uint64_t i = 0; i < n; ++i) host_out[i] = tmp[i];
  return ALTO_OK;
}

alto_status alto_slicer_destroy(alto_slicer* s) {
  if (s) {
    cudaDeviceSynchronize();  // batches may be in use on any stream
    delete s;
  }
  return ALTO_OK;
}

}  // extern "C"
