// C ABI entry points (include/alto_b200.h): argument checks, status codes,
// handle lifetimes.  The reference reports misuse with assert()/exit(); here
// every entry point validates its arguments and returns an alto_status.
#include <cstdarg>
#include <cstring>
#include <mutex>
#include <new>

#include "alto_internal.cuh"

namespace alto {

std::atomic<uint64_t> g_kernel_launches{0};
thread_local cudaStream_t tls_alloc_stream = nullptr;
static thread_local char g_err[512] = "";

cudaMemPool_t transient_pool() {
  static std::mutex mu;
  static cudaMemPool_t pools[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
  std::lock_guard<std::mutex> g(mu);
  if (!pools[dev]) {
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t p = nullptr;
    if (cudaMemPoolCreate(&p, &props) != cudaSuccess) return nullptr;
    uint64_t keep = ~0ull;  // keep freed memory for the next call
    cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep);
    pools[dev] = p;
  }
  return pools[dev];
}

void set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}

alto_status export_keys(const alto_tensor* t, uint64_t* d_out, float* d_vals, cudaStream_t st);

// Shape checks only (no index is read).
alto_status check_coo_shape(const alto_coo* coo) {
  if (!coo) {
    set_error("coo is NULL");
    return ALTO_ERR_INVALID;
  }
  if (coo->nmodes < 1 || coo->nmodes > ALTO_MAX_MODES) {
    set_error("nmodes %d outside 1..%d", coo->nmodes, ALTO_MAX_MODES);
    return ALTO_ERR_INVALID;
  }
  if (!coo->dims || (coo->nnz && (!coo->cidx || !coo->vals))) {
    set_error("coo dims/cidx/vals missing");
    return ALTO_ERR_INVALID;
  }
  if (coo->index_bytes != 8 && coo->index_bytes != 4) {
    set_error("index_bytes must be 4 or 8");
    return ALTO_ERR_INVALID;
  }
  if (coo->val_dtype != ALTO_F64 && coo->val_dtype != ALTO_F32) {
    set_error("values must be float64 or float32");
    return ALTO_ERR_INVALID;
  }
  if (coo->nnz >= (1ull << 32)) {
    set_error("nnz %llu exceeds 2^32-1", (unsigned long long)coo->nnz);
    return ALTO_ERR_UNSUPPORTED;
  }
  for (int m = 0; m < coo->nmodes; ++m) {
    if (coo->dims[m] < 1 || coo->dims[m] > 0xffffffffull) {
      set_error("dims[%d]=%llu outside 1..2^32-1", m, (unsigned long long)coo->dims[m]);
      return ALTO_ERR_INVALID;
    }
    if (coo->nnz && !coo->cidx[m]) {
      set_error("cidx[%d] is NULL", m);
      return ALTO_ERR_INVALID;
    }
  }
  return ALTO_OK;
}

static alto_status check_coo(const alto_coo* coo) {
  ALTO_TRY(check_coo_shape(coo));
  if (!coo->on_device) {  // host indices are checked against dims (the reference asserts)
    for (int m = 0; m < coo->nmodes; ++m) {
      for (uint64_t i = 0; i < coo->nnz; ++i) {
        uint64_t v = coo->index_bytes == 8 ? ((const uint64_t*)coo->cidx[m])[i]
                                           : ((const uint32_t*)coo->cidx[m])[i];
        if (v >= coo->dims[m]) {
          set_error("cidx[%d][%llu]=%llu >= dims[%d]=%llu", m, (unsigned long long)i,
                    (unsigned long long)v, m, (unsigned long long)coo->dims[m]);
          return ALTO_ERR_INVALID;
        }
      }
    }
  }
  return ALTO_OK;
}

static int bits_needed(const alto_coo* coo) {
  int b = 0;
  for (int m = 0; m < coo->nmodes; ++m)
    b += coo->dims[m] <= 1 ? 0 : 64 - __builtin_clzll(coo->dims[m] - 1);
  return b;
}

}  // namespace alto

using namespace alto;

extern "C" {

const char* alto_status_string(alto_status s) {
  switch (s) {
    case ALTO_OK: return "ok";
    case ALTO_ERR_INVALID: return "invalid argument";
    case ALTO_ERR_CUDA: return "CUDA error";
    case ALTO_ERR_NOMEM: return "out of device memory";
    case ALTO_ERR_NOT_SPD: return "matrix not positive definite";
    case ALTO_ERR_UNSUPPORTED: return "unsupported configuration";
    case ALTO_ERR_TIMEOUT: return "device wait timed out";
  }
  return "unknown status";
}

const char* alto_last_error(void) { return g_err; }
int alto_version(void) { return ALTO_VERSION; }
uint64_t alto_kernel_launches(void) { return g_kernel_launches.load(); }

alto_status alto_compute_masks(int nmodes, const uint64_t* dims, int key_bits, uint64_t* masks,
                               uint64_t* alto_mask, int* alto_bits) {
  if (nmodes < 1 || nmodes > ALTO_MAX_MODES || !dims) {
    set_error("bad nmodes or dims");
    return ALTO_ERR_INVALID;
  }
  if (key_bits != 64 && key_bits != 128) {
    set_error("key_bits must be 64 or 128");
    return ALTO_ERR_INVALID;
  }
  Key2 mk[ALTO_MAX_MODES], am;
  int bits[ALTO_MAX_MODES];
  int total = setup_masks(nmodes, dims, key_bits, mk, &am, bits);
  if (total < 0) {
    set_error("index bits exceed the %d-bit key", key_bits);
    return ALTO_ERR_UNSUPPORTED;
  }
  if (masks)
    for (int m = 0; m < nmodes; ++m) {
      masks[2 * m] = mk[m].lo;
      masks[2 * m + 1] = mk[m].hi;
    }
  if (alto_mask) {
    alto_mask[0] = am.lo;
    alto_mask[1] = am.hi;
  }
  if (alto_bits) *alto_bits = total;
  return ALTO_OK;
}

alto_status alto_tensor_create(const alto_coo* coo, int key_bits, int nprtn, int stream_mode,
                               alto_cuda_stream stream, alto_tensor** out) {
  if (!out) {
    set_error("out is NULL");
    return ALTO_ERR_INVALID;
  }
  *out = nullptr;
  ALTO_TRY(check_coo(coo));
  if (nprtn < 1) {
    set_error("nprtn must be >= 1");
    return ALTO_ERR_INVALID;
  }
  if (stream_mode >= coo->nmodes) {
    set_error("stream_mode %d >= nmodes", stream_mode);
    return ALTO_ERR_INVALID;
  }
  int need = bits_needed(coo);
  if (key_bits == 0) key_bits = need <= 64 ? 64 : 128;
  if (key_bits != 64 && key_bits != 128) {
    set_error("key_bits must be 0, 64 or 128");
    return ALTO_ERR_INVALID;
  }
  if (need > key_bits) {
    set_error("index bits %d exceed the %d-bit key", need, key_bits);
    return ALTO_ERR_UNSUPPORTED;
  }
  int dev = 0;
  ALTO_TRY_CUDA(cudaGetDevice(&dev));
  alto_tensor* t = new (std::nothrow) alto_tensor();
  if (!t) return ALTO_ERR_NOMEM;
  t->key_bits = key_bits;
  t->stream_mode = stream_mode < 0 ? -1 : stream_mode;
  t->stream = (cudaStream_t)stream;
  alto_status s = encode_tensor(t, coo, nprtn, (cudaStream_t)stream);
  if (s != ALTO_OK) {
    delete t;
    return s;
  }
  *out = t;
  return ALTO_OK;
}

alto_status alto_tensor_update(alto_tensor* t, const alto_coo* coo, int nprtn,
                               alto_cuda_stream stream) {
  if (!t) {
    set_error("tensor is NULL");
    return ALTO_ERR_INVALID;
  }
  ALTO_TRY(check_coo(coo));
  if (coo->nmodes != t->nmodes) {
    set_error("update has %d modes, tensor %d", coo->nmodes, t->nmodes);
    return ALTO_ERR_INVALID;
  }
  if (nprtn < 1) {
    set_error("nprtn must be >= 1");
    return ALTO_ERR_INVALID;
  }
  if (bits_needed(coo) > t->key_bits) {
    set_error("index bits exceed the %d-bit key", t->key_bits);
    return ALTO_ERR_UNSUPPORTED;
  }
  return encode_tensor(t, coo, nprtn, (cudaStream_t)stream);
}

alto_status alto_tensor_export(const alto_tensor* t, uint64_t* masks, uint64_t* alto_mask,
                               uint64_t* idx, double* vals, uint64_t* perm, uint64_t* prtn_ptr,
                               uint64_t* intervals) {
  if (!t) {
    set_error("tensor is NULL");
    return ALTO_ERR_INVALID;
  }
  cudaStream_t st = t->stream;
  const int N = t->nmodes;
  const uint64_t nnz = t->nnz;
  if (masks)
    for (int m = 0; m < N; ++m) {
      masks[2 * m] = t->masks[m].lo;
      masks[2 * m + 1] = t->masks[m].hi;
    }
  if (alto_mask) {
    alto_mask[0] = t->alto_mask.lo;
    alto_mask[1] = t->alto_mask.hi;
  }
  if (prtn_ptr)
    for (int p = 0; p <= t->nprtn; ++p) prtn_ptr[p] = t->prtn_ptr[p];
  if (intervals)
    ALTO_TRY_CUDA(cudaMemcpyAsync(intervals, t->prtn_iv.p, (size_t)t->nprtn * N * 2 * 8,
                                  cudaMemcpyDeviceToHost, st));
  if (nnz && (idx || vals || perm)) {
    DevBuf tmp, tmpv;
    ALTO_TRY(tmp.ensure(nnz * 16));
    ALTO_TRY(tmpv.ensure(nnz * 4));
    ALTO_TRY(export_keys(t, idx ? tmp.as<uint64_t>() : nullptr, tmpv.as<float>(), st));
    if (idx) ALTO_TRY_CUDA(cudaMemcpyAsync(idx, tmp.p, nnz * 16, cudaMemcpyDeviceToHost, st));
    if (vals) {
      std::vector<float> v(nnz);
      ALTO_TRY_CUDA(cudaMemcpyAsync(v.data(), tmpv.p, nnz * 4, cudaMemcpyDeviceToHost, st));
      ALTO_TRY_CUDA(cudaStreamSynchronize(st));
      for (uint64_t i = 0; i < nnz; ++i) vals[i] = v[i];
    }
    if (perm) {
      std::vector<uint32_t> p(nnz);
      ALTO_TRY_CUDA(cudaMemcpyAsync(p.data(), t->perm.p, nnz * 4, cudaMemcpyDeviceToHost, st));
      ALTO_TRY_CUDA(cudaStreamSynchronize(st));
      for (uint64_t i = 0; i < nnz; ++i) perm[i] = p[i];
    }
  }
  ALTO_TRY_CUDA(cudaStreamSynchronize(st));
  return ALTO_OK;
}

alto_status alto_tensor_info(const alto_tensor* t, int* nmodes, uint64_t* dims, uint64_t* nnz,
                             int* key_bits, int* alto_bits, int* nprtn, int* stream_mode) {
  if (!t) {
    set_error("tensor is NULL");
    return ALTO_ERR_INVALID;
  }
  if (nmodes) *nmodes = t->nmodes;
  if (dims)
    for (int m = 0; m < t->nmodes; ++m) dims[m] = t->dims[m];
  if (nnz) *nnz = t->nnz;
  if (key_bits) *key_bits = t->key_bits;
  if (alto_bits) *alto_bits = t->alto_bits;
  if (nprtn) *nprtn = t->nprtn;
  if (stream_mode) *stream_mode = t->stream_mode;
  return ALTO_OK;
}

alto_status alto_tensor_device_bytes(const alto_tensor* t, uint64_t* bytes) {
  if (!t || !bytes) {
    set_error("tensor or bytes is NULL");
    return ALTO_ERR_INVALID;
  }
  uint64_t b = t->line.bytes + t->perm.bytes + t->tile_iv.bytes + t->prtn_iv.bytes + t->scratch.bytes +
               t->scan_scratch.bytes + t->err.bytes;
  for (int m = 0; m < ALTO_MAX_MODES; ++m) b += t->sorted[m].line.bytes + t->sorted[m].tile_iv.bytes;
  *bytes = b;
  return ALTO_OK;
}

alto_status alto_tensor_restrict(alto_tensor* t, uint64_t begin, uint64_t end, alto_cuda_stream stream) {
  if (!t || begin > end || end > t->nnz) {
    set_error("bad tensor or range [%llu, %llu) of %llu entries", (unsigned long long)begin,
              (unsigned long long)end, t ? (unsigned long long)t->nnz : 0ull);
    return ALTO_ERR_INVALID;
  }
  return restrict_line(t, begin, end, (cudaStream_t)stream);
}

alto_status alto_tensor_destroy(alto_tensor* t) {
  delete t;
  return ALTO_OK;
}

static alto_status check_mttkrp(const alto_tensor* t, int mode, const void* const* factors,
                                alto_dtype fdtype, int rank, const float* out) {
  if (!t || !factors || !out) {
    set_error("tensor, factors or out is NULL");
    return ALTO_ERR_INVALID;
  }
  if (mode < 0 || mode >= t->nmodes) {
    set_error("mode %d outside 0..%d", mode, t->nmodes - 1);
    return ALTO_ERR_INVALID;
  }
  if (rank < 1) {
    set_error("rank must be >= 1");
    return ALTO_ERR_INVALID;
  }
  if (fdtype != ALTO_F32 && fdtype != ALTO_BF16) {
    set_error("factor dtype must be float32 or bfloat16");
    return ALTO_ERR_INVALID;
  }
  for (int m = 0; m < t->nmodes; ++m)
    if (m != mode && !factors[m]) {
      set_error("factors[%d] is NULL", m);
      return ALTO_ERR_INVALID;
    }
  return ALTO_OK;
}

alto_status alto_mttkrp(alto_tensor* t, int mode, const void* const* factors, alto_dtype fdtype,
                        int rank, float* out, int accumulate, alto_cuda_stream stream) {
  ALTO_TRY(check_mttkrp(t, mode, factors, fdtype, rank, out));
  return run_mttkrp(t, mode, factors, fdtype, rank, out, accumulate, ALTO_MTTKRP_AUTO,
                    (cudaStream_t)stream);
}

alto_status alto_mttkrp_variant_run(alto_tensor* t, int mode, const void* const* factors,
                                    alto_dtype fdtype, int rank, float* out, int accumulate,
                                    alto_mttkrp_variant variant, alto_cuda_stream stream) {
  ALTO_TRY(check_mttkrp(t, mode, factors, fdtype, rank, out));
  const int bulk = ((int)variant & ALTO_MTTKRP_FEED_BULK) ? 1 : 0;
  const int dense = ((int)variant & ALTO_MTTKRP_FEED_DENSE) ? 1 : 0;
  const int fixed = ((int)variant & ALTO_MTTKRP_FEED_FIXED_TARGET) ? 1 : 0;
  const alto_mttkrp_variant v = (alto_mttkrp_variant)(
      (int)variant & ~(ALTO_MTTKRP_FEED_BULK | ALTO_MTTKRP_FEED_DENSE | ALTO_MTTKRP_FEED_FIXED_TARGET));
  if (v < ALTO_MTTKRP_AUTO || v > ALTO_MTTKRP_DETERMINISTIC || bulk + dense + fixed > 1 ||
      (bulk && v != ALTO_MTTKRP_ATOMIC && v != ALTO_MTTKRP_SORTED) ||
      ((dense || fixed) && (v != ALTO_MTTKRP_SORTED || t->nmodes != 3))) {
    set_error("unknown variant %d", (int)variant);
    return ALTO_ERR_INVALID;
  }
  return run_mttkrp_feed(t, mode, factors, fdtype, rank, out, accumulate, v,
                         v == ALTO_MTTKRP_AUTO ? -1 : (fixed ? 3 : dense ? 2 : bulk), (cudaStream_t)stream);
}

alto_status alto_mttkrp_autotune(alto_tensor* t, const void* const* factors, alto_dtype fdtype,
                                 int rank, alto_cuda_stream stream, alto_mttkrp_variant* variants) {
  if (!t || !factors || rank < 1 || (fdtype != ALTO_F32 && fdtype != ALTO_BF16)) {
    set_error("bad arguments");
    return ALTO_ERR_INVALID;
  }
  for (int m = 0; m < t->nmodes; ++m)
    if (!factors[m]) {
      set_error("factors[%d] is NULL", m);
      return ALTO_ERR_INVALID;
    }
  return autotune(t, factors, fdtype, rank, (cudaStream_t)stream, variants);
}

alto_status alto_mttkrp_choose(const alto_tensor* t, int mode, int rank, alto_dtype fdtype,
                               alto_mttkrp_variant* variant) {
  if (!t || !variant || mode < 0 || mode >= t->nmodes) {
    set_error("bad arguments");
    return ALTO_ERR_INVALID;
  }
  *variant = choose_variant(t, mode, rank, fdtype);
  return ALTO_OK;
}

}  // extern "C"
