// cpd64 -- the reference's command-line driver (src/main.cpp), rebuilt on the
// C ABI of libalto_b200 so that every MTTKRP, CP-ALS and CP-stream step runs
// on the GPU.  Flags follow src/main.cpp:68-93:
//
//   -i FILE   .tns text tensor (1-based unless -u)      -b FILE  binary tensor
//   -r R      rank (16)                                 -m K     max iterations (10)
//   -x SEED   seed for the initial model (srand/rand)   -t MODE  target mode (-1: all)
//   -e EPS    epsilon (5e-2)                            -u       zero-based indices
//   -p        MTTKRP benchmark (BenchmarkAlto)          -c       check MTTKRP against COO
//   -l MODEL  als | cpstream_alto                       -z CON   nonneg | lasso
//   -a MODE   streaming mode                            -g L     time slices per batch (1)
//   -k T      nonzero threshold per batch               -f N     save to file (0): N != 0
//                                                                writes a text input back as
//                                                                binary, a binary input as text
//   -o FILE   output file: the tensor read, as text (the reference parses -o but
//             its only use is commented out, src/main.cpp:152-153, 355)
//   -d/-s     dims / sparsity of a generated tensor: parsed, then refused (the
//             reference's Poisson generator is not part of this library)
//   --forgetting F   CP-stream forgetting factor (0.99; the reference fixes it
//                    at compile time, src/streaming_cpd.cpp:18); long form only
//   -h / -v   help / version
//
// The initial model uses the C library's rand() after srand(seed), drawing
// values in [-3, 3] with a random sign as the reference does
// (src/util.cpp:28-43, src/main.cpp:188), so both drivers start from the
// same model on the same C library.  -c computes its float64 COO ground
// truth on the host: it is a verification mode, as in the reference.
#include <getopt.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "alto_b200.h"

namespace {

// The tensor's shape, and (for --check only) a host copy of its nonzeros.
struct Coo {
  int nmodes = 0;
  uint64_t count = 0;
  std::vector<uint64_t> dims;
  std::vector<std::vector<uint64_t>> cidx;
  std::vector<double> vals;
  uint64_t nnz() const { return count; }
};

[[noreturn]] void die(const char* what, alto_status s) {
  fprintf(stderr, "cpd64: %s failed: %s (%s)\n", what, alto_status_string(s), alto_last_error());
  exit(1);
}

#define CHECK(call)                   \
  do {                                \
    alto_status s_ = (call);          \
    if (s_ != ALTO_OK) die(#call, s_); \
  } while (0)

// rand_val of the reference (src/util.cpp:28-35).
double rand_val() {
  double v = 3.0 * ((double)rand() / (double)RAND_MAX);
  if (rand() % 2 == 0) v *= -1;
  return v;
}

std::vector<std::vector<double>> random_model(const std::vector<uint64_t>& dims, int R) {
  std::vector<std::vector<double>> U(dims.size());
  for (size_t m = 0; m < dims.size(); ++m) {
    U[m].resize(dims[m] * R);
    for (auto& x : U[m]) x = rand_val();
  }
  return U;
}

double now() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

void usage(const char* argv0) {
  fprintf(stderr,
          "usage: %s (-i FILE | -b FILE) [-r R] [-m K] [-x SEED] [-t MODE] [-e EPS] [-u]\n"
          "          [-p | -c | -l als|cpstream_alto|spcpstream_alto] [-z nonneg|lasso] [-a MODE]\n"
          "          [-g L] [-k T] [-f N] [-o FILE] [--forgetting F]\n",
          argv0);
}

int run_bench(alto_tensor* t, const Coo& X, int R, int target, int iters) {
  auto U = random_model(X.dims, R);
  std::vector<double*> ptrs(X.nmodes);
  for (int m = 0; m < X.nmodes; ++m) ptrs[m] = U[m].data();
  int m0 = target < 0 ? 0 : target, m1 = target < 0 ? X.nmodes : target + 1;
  for (int m = m0; m < m1; ++m) CHECK(alto_mttkrp_host(t, m, ptrs.data(), R, nullptr));
  double t0 = now();
  for (int i = 0; i < iters; ++i)
    for (int m = m0; m < m1; ++m) CHECK(alto_mttkrp_host(t, m, ptrs.data(), R, nullptr));
  printf("ALTO runtime:   %f\n", now() - t0);
  return 0;
}

int run_check(alto_tensor* t, const Coo& X, int R, int target) {
  auto U = random_model(X.dims, R);
  int m0 = target < 0 ? 0 : target, m1 = target < 0 ? X.nmodes : target + 1;
  int bad_modes = 0;
  for (int mode = m0; mode < m1; ++mode) {
    std::vector<std::vector<double>> F = U;
    std::fill(F[mode].begin(), F[mode].end(), 0.0);
    std::vector<double> truth(X.dims[mode] * R, 0.0), row(R);
    for (uint64_t i = 0; i < X.nnz(); ++i) {  // COO ground truth (src/mttkrp.cpp:122-156)
      for (int r = 0; r < R; ++r) row[r] = X.vals[i];
      for (int m = 0; m < X.nmodes; ++m)
        if (m != mode)
          for (int r = 0; r < R; ++r) row[r] *= F[m][X.cidx[m][i] * R + r];
      for (int r = 0; r < R; ++r) truth[X.cidx[mode][i] * R + r] += row[r];
    }
    std::vector<double*> ptrs(X.nmodes);
    for (int m = 0; m < X.nmodes; ++m) ptrs[m] = F[m].data();
    CHECK(alto_mttkrp_host(t, mode, ptrs.data(), R, nullptr));
    double maxabs = 0, maxerr = 0;
    for (size_t q = 0; q < truth.size(); ++q) {
      maxabs = std::max(maxabs, std::fabs(truth[q]));
      maxerr = std::max(maxerr, std::fabs(truth[q] - F[mode][q]));
    }
    const double rel = maxabs > 0 ? maxerr / maxabs : maxerr;
    printf("mode %d: normwise error %.3e %s\n", mode, rel, rel <= 1e-5 ? "correct" : "INCORRECT");
    bad_modes += rel > 1e-5;
  }
  return bad_modes ? 1 : 0;
}

int run_als(alto_tensor* t, const Coo& X, int R, int iters, double eps) {
  auto U = random_model(X.dims, R);
  std::vector<double> lambda(R, 1.0), fits(std::max(iters, 1));
  std::vector<double*> ptrs(X.nmodes);
  for (int m = 0; m < X.nmodes; ++m) ptrs[m] = U[m].data();
  printf("Running ALTO CP-ALS with %d max iterations and %.2e epsilon\n", iters, eps);
  int done = 0;
  double t0 = now();
  CHECK(alto_cpd_als(t, R, ptrs.data(), lambda.data(), iters, eps, ALTO_FIT_REFERENCE, ALTO_F32,
                     fits.data(), &done, nullptr));
  double el = now() - t0;
  for (int i = 0; i < done; ++i)
    printf("it: %d\t fit: %g\t fit-delta: %g\n", i, fits[i], i ? std::fabs(fits[i] - fits[i - 1]) : fits[i]);
  printf("CPD (ALTO) time: %f s (%d iterations)\n", el, done);
  return 0;
}

// StreamingSparseTensor (src/streaming_sptensor.cpp:69-264) on the device
// (alto_slicer_*): sort by the stream mode then the following modes
// cyclically, relabel the non-stream indices in first-seen order, and cut
// batches of timeslice_limit time steps (or until nnz_threshold); each batch
// goes to the session as it lies in device memory.
int run_cpstream(const alto_coo& in, int R, int iters, double eps, int tmode, alto_constraint con, bool sparse,
                 uint64_t nnz_threshold, uint64_t limit, double forgetting) {
  const int N = in.nmodes;
  alto_slicer* sl = nullptr;
  CHECK(alto_slicer_create(&in, tmode, nullptr, &sl));
  alto_stream_session* s = nullptr;
  CHECK(alto_stream_open(N, tmode, R, con, forgetting, iters, eps, nullptr, &s));
  if (sparse) CHECK(alto_stream_set_model(s, ALTO_MODEL_SPCPSTREAM));
  int nb = 0;
  double t0 = now();
  for (;;) {
    alto_coo B;
    int got = 0;
    CHECK(alto_slicer_next(sl, nnz_threshold, limit, &B, &got));
    if (!got) break;
    if (B.nnz == 0) continue;
    std::vector<double> init;
    static std::vector<uint64_t> have(ALTO_MAX_MODES, 0);
    for (int m = 0; m < N; ++m) {
      uint64_t d = std::max(have[m], B.dims[m]);
      for (uint64_t q = have[m] * R; q < d * R; ++q) init.push_back(rand_val());
      have[m] = d;
    }
    int inner = 0;
    CHECK(alto_stream_push(s, &B, init.data(), init.size(), &inner));
    ++nb;
    fprintf(stderr, "batch %d: %llu nnz, %d inner iterations\n", nb, (unsigned long long)B.nnz, inner);
  }
  double el = now() - t0;
  printf("%s (ALTO) on the GPU: %d batches in %f s (%f s/batch)\n", sparse ? "spCPSTREAM" : "CPSTREAM", nb, el,
         nb ? el / nb : 0.0);
  // cpd_error of the final model against the whole (relabelled) tensor, as
  // the reference reports it (src/streaming_cpd.cpp:311-345)
  alto_coo whole;
  double err = 0;
  CHECK(alto_slicer_tensor(sl, &whole));
  if (nb && alto_stream_error(s, &whole, &err) == ALTO_OK) printf("final fit error: %f\n", err * err);
  alto_stream_close(s);
  alto_slicer_destroy(sl);
  return 0;
}

// getopt code of the long-only --forgetting option (no short letter: -f is
// the reference's --file)
constexpr int kForgettingOpt = 0x100;

}  // namespace

int main(int argc, char** argv) {
  static const option long_opt[] = {
      {"help", 0, nullptr, 'h'}, {"version", 0, nullptr, 'v'}, {"input", 1, nullptr, 'i'},
      {"bin", 1, nullptr, 'b'}, {"model", 1, nullptr, 'l'}, {"constraint", 1, nullptr, 'z'},
      {"rank", 1, nullptr, 'r'}, {"max-iter", 1, nullptr, 'm'}, {"seed", 1, nullptr, 'x'},
      {"target-mode", 1, nullptr, 't'}, {"epsilon", 1, nullptr, 'e'}, {"zero-based", 0, nullptr, 'u'},
      {"check", 0, nullptr, 'c'}, {"bench", 0, nullptr, 'p'}, {"streaming-mode", 1, nullptr, 'a'},
      {"timeslice-limit", 1, nullptr, 'g'}, {"nnz-threshold", 1, nullptr, 'k'},
      {"file", 1, nullptr, 'f'}, {"output", 1, nullptr, 'o'}, {"dims", 1, nullptr, 'd'},
      {"sparsity", 1, nullptr, 's'}, {"forgetting", 1, nullptr, kForgettingOpt}, {nullptr, 0, nullptr, 0}};
  std::string text, bin, out_file, model = "als";
  int R = 16, iters = 10, target = -1, tmode = -1, save_to_file = 0;
  bool generate = false;
  double eps = 5e-2, forgetting = 0.99;
  bool zero = false, check = false, bench = false;
  alto_constraint con = ALTO_UNCONSTRAINED;
  uint64_t nnz_threshold = UINT64_MAX, limit = 1;
  srand((unsigned)time(nullptr));
  int c;
  // the reference's short options (src/main.cpp:93)
  while ((c = getopt_long(argc, argv, "hvi:o:b:l:z:r:m:x:d:t:s:e:f:ucpa:g:k:", long_opt, nullptr)) != -1) {
    switch (c) {
      case 'h': usage(argv[0]); return 0;
      case 'v': printf("cpd64 (B200) %d\n", alto_version()); return 0;
      case 'i': text = optarg; break;
      case 'b': bin = optarg; break;
      case 'l': model = optarg; break;
      case 'z':
        if (!strcmp(optarg, "nonneg")) con = ALTO_NONNEG;
        else if (!strcmp(optarg, "lasso")) con = ALTO_LASSO;
        break;
      case 'r': R = atoi(optarg); break;
      case 'm': iters = atoi(optarg); break;
      case 'x': srand((unsigned)atoi(optarg)); break;
      case 't': target = atoi(optarg); break;
      case 'e': eps = atof(optarg); break;
      case 'u': zero = true; break;
      case 'c': check = true; break;
      case 'p': bench = true; break;
      case 'a': tmode = atoi(optarg); break;
      case 'g': limit = strtoull(optarg, nullptr, 10); break;
      case 'k': nnz_threshold = strtoull(optarg, nullptr, 10); break;
      case 'f':
        save_to_file = atoi(optarg);
        if (save_to_file < 0) fprintf(stderr, "Invalid -file: %s.\n", optarg);
        break;
      case 'o': out_file = optarg; break;
      case 'd':
      case 's': generate = true; break;
      case kForgettingOpt: forgetting = atof(optarg); break;
      default: usage(argv[0]); return 1;
    }
  }
  if (generate && bin.empty() && text.empty()) {
    fprintf(stderr, "cpd64: generated tensors (-d/-s) are not supported here; pass -i or -b\n");
    return 1;
  }
  // ImportSparseTensor (src/sptensor.cpp:160-249), parsed on the device
  if (bin.empty() && text.empty()) {
    usage(argv[0]);
    return 1;
  }
  const std::string& path = bin.empty() ? text : bin;
  alto_dcoo* D = nullptr;
  if (alto_read_tensor(path.c_str(), bin.empty() ? ALTO_FILE_TEXT : ALTO_FILE_BINARY, zero ? 1 : 0, nullptr, &D) !=
      ALTO_OK) {
    fprintf(stderr, "cannot read %s: %s\n", path.c_str(), alto_last_error());
    return 1;
  }
  alto_coo coo;
  CHECK(alto_dcoo_view(D, &coo));
  // -f: the reference writes the tensor back in the other format under its
  // own file name (src/main.cpp:268-289, ExportSparseTensor with path NULL,
  // src/sptensor.cpp:33-45)
  if (save_to_file) {
    const bool to_text = !bin.empty();
    char fn[64];
    snprintf(fn, sizeof fn, "%lluD_%llu.%s", (unsigned long long)coo.nmodes, (unsigned long long)coo.nnz,
             to_text ? "tns" : "bin");
    double tw = now();
    CHECK(alto_write_tensor(fn, to_text ? ALTO_FILE_TEXT : ALTO_FILE_BINARY, &coo));
    printf("Writing to %s file: %f\n", to_text ? "text" : "binary", now() - tw);
  }
  if (!out_file.empty()) CHECK(alto_write_tensor(out_file.c_str(), ALTO_FILE_TEXT, &coo));
  Coo X;
  X.nmodes = coo.nmodes;
  X.count = coo.nnz;
  X.dims.assign(coo.dims, coo.dims + coo.nmodes);
  if (check) {  // host copy for the COO ground truth
    std::vector<uint64_t> flat((size_t)X.nmodes * X.count);
    X.vals.resize(X.count);
    CHECK(alto_dcoo_to_host(D, flat.data(), X.vals.data()));
    for (int m = 0; m < X.nmodes; ++m)
      X.cidx.emplace_back(flat.begin() + (size_t)m * X.count, flat.begin() + (size_t)(m + 1) * X.count);
  }
  if (R < 1 || target >= X.nmodes) { usage(argv[0]); return 1; }
  printf("tensor: %d modes, %llu nonzeros, rank %d\n", X.nmodes, (unsigned long long)X.nnz(), R);
  if (model == "cpstream_alto" || model == "CPSTREAM_ALTO") {
    if (tmode < 0 || tmode >= X.nmodes) { fprintf(stderr, "need -a streaming mode\n"); return 1; }
    return run_cpstream(coo, R, iters, eps, tmode, con, false, nnz_threshold, limit ? limit : 1, forgetting);
  }
  if (model == "spcpstream_alto" || model == "SPCPSTREAM_ALTO") {
    if (tmode < 0 || tmode >= X.nmodes) { fprintf(stderr, "need -a streaming mode\n"); return 1; }
    return run_cpstream(coo, R, iters, eps, tmode, con, true, nnz_threshold, limit ? limit : 1, forgetting);
  }
  alto_tensor* t = nullptr;
  double t0 = now();
  CHECK(alto_tensor_create(&coo, 0, 1, -1, nullptr, &t));
  printf("ALTO creation time:   %f\n", now() - t0);
  int rc = 0;
  if (check) rc = run_check(t, X, R, target);
  else if (bench) rc = run_bench(t, X, R, target, iters);
  else rc = run_als(t, X, R, iters, eps);
  alto_tensor_destroy(t);
  alto_dcoo_destroy(D);
  return rc;
}
