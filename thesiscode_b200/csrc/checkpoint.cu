// Checkpoint and restart of the device-resident RK4 state (tc_rk4_save,
// tc_rk4_restore).
//
// The reference keeps no restart files: its drivers write VTK frames and a
// final data table only (RHWavePanelsMPI.f90:327-333). A long run on the
// device can instead be stopped and continued. The file holds what the next
// step needs and nothing else:
//   * positions of the three target classes;
//   * active vorticity and areas;
//   * Omega and the three deltas;
//   * for a forced (stratosphere) run, the absolute vorticity and the clock:
//     t0, step count and step length, kept apart so the stage times round
//     exactly as in an uninterrupted run.
// A restored context therefore continues bit for bit as the run that wrote
// the file would have.
//
// Layout (little-endian, as on every host this library builds for):
//   char[8] "TCB2RK4" + NUL; u32 version (1); u32 flags (bit 0: forced run);
//   i32 nA, nV, nQ, precision; i64 steps since load, forced step count;
//   f64 Omega, delta[3], t0, forced step length;
//   f64 xA[3nA], zetaA[nA], areaA[nA], xV[3nV], xQ[3nQ];
//   forced runs also f64 absVortA[nA], absVortV[nV];
//   u64 FNV-1a hash of every byte before it.
// tc_rk4_save writes `path`.tmp and renames it over `path`, so a crash in the
// middle leaves the previous checkpoint whole.
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "tc_ctx.h"

namespace {

constexpr char kMagic[8] = {'T', 'C', 'B', '2', 'R', 'K', '4', '\0'};
constexpr uint32_t kVersion = 1;

struct Header {
  char magic[8];
  uint32_t version, flags;
  int32_t nA, nV, nQ, precision;
  int64_t steps, strat_step;
  double omega, delta[3], t0, strat_dt;
};
static_assert(sizeof(Header) == 96, "checkpoint header layout");

uint64_t fnv1a(const unsigned char* p, size_t n, uint64_t h = 1469598103934665603ull) {
  for (size_t i = 0; i < n; ++i) {
    h ^= p[i];
    h *= 1099511628211ull;
  }
  return h;
}

// The arrays of a checkpoint, in file order: (device buffer, doubles).
struct Section {
  tcb::DevBuf* buf;
  size_t count;
};

std::vector<Section> sections(tcb::Rk4State& R, bool forced) {
  std::vector<Section> s = {{&R.x0A, 3 * (size_t)R.nA}, {&R.z0, (size_t)R.nA},
                            {&R.areaA, (size_t)R.nA},   {&R.x0V, 3 * (size_t)R.nV},
                            {&R.x0Q, 3 * (size_t)R.nQ}};
  if (forced) {
    s.push_back({&R.absA, (size_t)R.nA});
    s.push_back({&R.absV, (size_t)R.nV});
  }
  return s;
}

}  // namespace

extern "C" int tc_rk4_save(tc_ctx* ctx, const char* path) {
  if (!ctx || !path) return TC_ERR_ARG;
  if (cudaSetDevice(ctx->device) != cudaSuccess) {
    tc_record_error("tc_rk4_save: cudaSetDevice(%d) failed", ctx->device);
    return TC_ERR_CUDA;
  }
  tcb::Rk4State& R = ctx->rk;
  if (!R.ready) {
    tc_record_error("tc_rk4_save: no RK4 state loaded");
    return TC_ERR_STATE;
  }
  Header h{};
  memcpy(h.magic, kMagic, sizeof(kMagic));
  h.version = kVersion;
  h.flags = R.strat ? 1u : 0u;
  h.nA = R.nA;
  h.nV = R.nV;
  h.nQ = R.nQ;
  h.precision = ctx->precision;
  h.steps = R.steps_total;
  h.strat_step = R.step;
  h.omega = ctx->omega;
  for (int c = 0; c < 3; ++c) h.delta[c] = ctx->delta[c];
  h.t0 = R.t0;
  h.strat_dt = R.strat_dt;
  std::vector<unsigned char> bytes(sizeof(Header));
  memcpy(bytes.data(), &h, sizeof(Header));
  for (const Section& s : sections(R, R.strat)) {
    const size_t off = bytes.size(), nb = s.count * sizeof(double);
    bytes.resize(off + nb);
    if (nb)
      TC_CUDA_TRY(cudaMemcpyAsync(bytes.data() + off, s.buf->ptr, nb, cudaMemcpyDeviceToHost,
                                  ctx->stream));
  }
  TC_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  const uint64_t sum = fnv1a(bytes.data(), bytes.size());
  const std::string tmp = std::string(path) + ".tmp";
  FILE* f = fopen(tmp.c_str(), "wb");
  if (!f) {
    tc_record_error("tc_rk4_save: cannot open %s for writing", tmp.c_str());
    return TC_ERR_ARG;
  }
  const bool ok = fwrite(bytes.data(), 1, bytes.size(), f) == bytes.size() &&
                  fwrite(&sum, sizeof(sum), 1, f) == 1;
  if (fclose(f) != 0 || !ok || rename(tmp.c_str(), path) != 0) {
    remove(tmp.c_str());
    tc_record_error("tc_rk4_save: writing %s failed", path);
    return TC_ERR_ARG;
  }
  return TC_OK;
}

// Reads and validates a checkpoint: magic, version, sizes against the file
// length, checksum. On success *h is its header and bytes its whole content.
static int read_checkpoint(const char* path, Header* h, std::vector<unsigned char>& bytes);

extern "C" int tc_rk4_checkpoint_info(const char* path, int* nA, int* nV, int* nQ, int* forced,
                                      long long* steps) {
  if (!path) return TC_ERR_ARG;
  Header h;
  std::vector<unsigned char> bytes;
  const int rc = read_checkpoint(path, &h, bytes);
  if (rc) return rc;
  if (nA) *nA = h.nA;
  if (nV) *nV = h.nV;
  if (nQ) *nQ = h.nQ;
  if (forced) *forced = (int)(h.flags & 1u);
  if (steps) *steps = h.steps;
  return TC_OK;
}

static int read_checkpoint(const char* path, Header* hp, std::vector<unsigned char>& bytes) {
  FILE* f = fopen(path, "rb");
  if (!f) {
    tc_record_error("checkpoint: cannot open %s", path);
    return TC_ERR_ARG;
  }
  bytes.clear();
  unsigned char chunk[1 << 16];
  size_t got;
  while ((got = fread(chunk, 1, sizeof(chunk), f)) > 0)
    bytes.insert(bytes.end(), chunk, chunk + got);
  fclose(f);
  Header h;
  if (bytes.size() < sizeof(Header) + sizeof(uint64_t)) {
    tc_record_error("checkpoint: %s is too short for a checkpoint", path);
    return TC_ERR_ARG;
  }
  memcpy(&h, bytes.data(), sizeof(Header));
  if (memcmp(h.magic, kMagic, sizeof(kMagic)) != 0 || h.version != kVersion || (h.flags & ~1u)) {
    tc_record_error("checkpoint: %s is not a version-%u checkpoint", path, kVersion);
    return TC_ERR_ARG;
  }
  const bool forced = (h.flags & 1u) != 0;
  if (h.nA < 0 || h.nV < 0 || h.nQ < 0) {
    tc_record_error("checkpoint: negative sizes in %s", path);
    return TC_ERR_ARG;
  }
  const size_t nA = (size_t)h.nA, nV = (size_t)h.nV, nQ = (size_t)h.nQ;
  const size_t doubles = 3 * nA + nA + nA + 3 * nV + 3 * nQ + (forced ? nA + nV : 0);
  const size_t body = bytes.size() - sizeof(Header) - sizeof(uint64_t);
  if (body != doubles * sizeof(double)) {
    tc_record_error("checkpoint: %s holds %zu bytes of arrays, its header asks for %zu", path,
                    body, doubles * sizeof(double));
    return TC_ERR_ARG;
  }
  uint64_t sum;
  memcpy(&sum, bytes.data() + bytes.size() - sizeof(sum), sizeof(sum));
  if (fnv1a(bytes.data(), bytes.size() - sizeof(sum)) != sum) {
    tc_record_error("checkpoint: %s fails its checksum", path);
    return TC_ERR_ARG;
  }
  *hp = h;
  return TC_OK;
}

extern "C" int tc_rk4_restore(tc_ctx* ctx, const char* path) {
  if (!ctx || !path) return TC_ERR_ARG;
  Header h;
  std::vector<unsigned char> bytes;
  int rc = read_checkpoint(path, &h, bytes);
  if (rc) return rc;
  const bool forced = (h.flags & 1u) != 0;
  const size_t nA = (size_t)h.nA, nV = (size_t)h.nV, nQ = (size_t)h.nQ;
  const size_t doubles = 3 * nA + nA + nA + 3 * nV + 3 * nQ + (forced ? nA + nV : 0);
  // the arrays, copied out of the byte buffer (which need not be 8-byte aligned)
  std::vector<double> a(doubles);
  memcpy(a.data(), bytes.data() + sizeof(Header), doubles * sizeof(double));
  const double* xA = a.data();
  const double* zA = xA + 3 * nA;
  const double* arA = zA + nA;
  const double* xV = arA + nA;
  const double* xQ = xV + 3 * nV;
  const double* absA = xQ + 3 * nQ;
  const double* absV = absA + nA;
  rc = tc_rk4_load(ctx, xA, zA, arA, h.nA, xV, h.nV, xQ, h.nQ, 0);
  if (rc) return rc;
  tcb::Rk4State& R = ctx->rk;
  if (forced) {
    const size_t D = sizeof(double);
    cudaError_t e = cudaSuccess;
    if ((rc = R.absA.ensure(std::max<size_t>(nA, 1) * D)) ||
        (rc = R.absV.ensure(std::max<size_t>(nV, 1) * D))) {
      cudaStreamSynchronize(ctx->stream);
      R.ready = false;
      return rc;
    }
    if (nA) e = cudaMemcpyAsync(R.absA.ptr, absA, nA * D, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess && nV)
      e = cudaMemcpyAsync(R.absV.ptr, absV, nV * D, cudaMemcpyHostToDevice, ctx->stream);
    if (e != cudaSuccess) {
      tc_record_cuda_error(e, "cudaMemcpyAsync (absolute vorticity)", __FILE__, __LINE__);
      cudaStreamSynchronize(ctx->stream);
      R.ready = false;
      return TC_ERR_CUDA;
    }
  }
  // the host arrays go out of scope at return
  TC_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  R.strat = forced;
  R.t0 = h.t0;
  R.step = h.strat_step;
  R.strat_dt = h.strat_dt;
  R.steps_total = h.steps;
  ctx->omega = h.omega;
  for (int c = 0; c < 3; ++c) ctx->delta[c] = h.delta[c];
  return TC_OK;
}

extern "C" int tc_rk4_steps_done(tc_ctx* ctx, long long* steps) {
  if (!ctx || !steps) return TC_ERR_ARG;
  if (!ctx->rk.ready) {
    tc_record_error("tc_rk4_steps_done: no RK4 state loaded");
    return TC_ERR_STATE;
  }
  *steps = ctx->rk.steps_total;
  return TC_OK;
}
