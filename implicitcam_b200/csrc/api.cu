// The C ABI of include/icam_cuda.h: pack creation and upload, point and brick reads,
// and the level bake of the brick cache, all on one CUDA stream per pack.
#include <cuda_runtime.h>

#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include <cub/cub.cuh>

#include "../../include/icam_cuda.h"
#include "kernels.h"
#include "pack_build.h"
#include "pack_state.h"

using namespace icam;

namespace {

int fail(IcamPack* pk, int code, const std::string& msg) {
  if (pk) pk->err = msg;
  return code;
}

#define CK(call)                                                                              \
  do {                                                                                        \
    cudaError_t e_ = (call);                                                                  \
    if (e_ != cudaSuccess) return fail(pk, ICAM_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

template <class T>
int upload(IcamPack* pk, const std::vector<T>& v, const T** out) {
  if (v.empty()) {
    *out = nullptr;
    return ICAM_OK;
  }
  void* d = nullptr;
  CK(cudaMalloc(&d, v.size() * sizeof(T)));
  pk->owned.push_back(d);
  CK(cudaMemcpyAsync(d, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, pk->stream));
  *out = static_cast<const T*>(d);
  return ICAM_OK;
}

// A scratch buffer of at least `bytes`, slot k.
int scratch(IcamPack* pk, int k, size_t bytes, void** out) {
  auto& b = pk->scratch[k];
  if (b.n < bytes) {
    if (b.p) CK(cudaFree(b.p));
    b.p = nullptr;
    b.n = 0;
    size_t want = std::max(bytes, size_t(1) << 16);
    CK(cudaMalloc(&b.p, want));
    b.n = want;
  }
  *out = b.p;
  return ICAM_OK;
}

// ICAM_MIXED_LEARNED: the seed network's starts for the brick kernel (it must have been
// trained or loaded on this pack).
int learned_starts(IcamPack* pk, int precision, BrickArgs* a) {
  if (precision != ICAM_MIXED_LEARNED) return ICAM_OK;
  if (pk->dev.n_subs == 0) return ICAM_OK;  // no B-spline sub-patch to seed: ICAM_MIXED
  if (!pk->net.ready)
    return fail(pk, ICAM_ERR_ARG, "ICAM_MIXED_LEARNED: train (icam_seednet_train) or load the seed network first");
  a->net_feat = pk->net.feat;
  a->net_w = pk->net.wbf;
  return ICAM_OK;
}

int grid_for(int64_t n, int threads) {
  int64_t g = (n + threads - 1) / threads;
  return int(std::max<int64_t>(1, std::min<int64_t>(g, 148 * 32)));
}

}  // namespace

extern "C" {

int icam_pack_create(const IcamSolidDesc* solid, const IcamPackOptions* opt, IcamPack** out, char* err,
                     size_t errlen) {
  auto report = [&](const std::string& m) {
    if (err && errlen) {
      std::snprintf(err, errlen, "%s", m.c_str());
    }
  };
  if (!solid || !out) {
    report("null argument");
    return ICAM_ERR_ARG;
  }
  *out = nullptr;
  IcamPack* pk = new IcamPack();
  pk->device = opt ? opt->device : 0;
  double need = opt && opt->need > 0 ? opt->need : 2.0;
  std::string e;
  if (!build_pack(solid, need, &pk->host, &e)) {
    report(e);
    delete pk;
    return ICAM_ERR_PACK;
  }
  int rc = ICAM_OK;
  auto cuda = [&](cudaError_t c, const char* what) {
    if (c != cudaSuccess && rc == ICAM_OK) {
      rc = ICAM_ERR_CUDA;
      report(std::string(what) + ": " + cudaGetErrorString(c));
    }
  };
  cuda(cudaSetDevice(pk->device), "cudaSetDevice");
  if (rc == ICAM_OK) cuda(cudaStreamCreateWithFlags(&pk->stream, cudaStreamNonBlocking), "cudaStreamCreate");
  if (rc != ICAM_OK) {
    delete pk;
    return rc;
  }
  HostPack& H = pk->host;
  DPack& D = pk->dev;
  int u = ICAM_OK;
  u |= upload(pk, H.faces, &D.faces);
  u |= upload(pk, H.nurbs, &D.nurbs);
  u |= upload(pk, H.subs, &D.subs);
  u |= upload(pk, H.sub_cp, &D.sub_cp);
  u |= upload(pk, H.sub_cp32, &D.sub_cp32);
  u |= upload(pk, H.span_cp, &D.span_cp);
  u |= upload(pk, H.breaks, &D.breaks);
  u |= upload(pk, H.edges, &D.edges);
  u |= upload(pk, H.pieces, &D.pieces);
  u |= upload(pk, H.verts, &D.verts);
  u |= upload(pk, H.cells, &D.cells);
  u |= upload(pk, H.insts, &D.insts);
  u |= upload(pk, H.among, &D.among);
  u |= upload(pk, H.tpieces, &D.tpieces);
  u |= upload(pk, H.bvh, &D.bvh);
  u |= upload(pk, H.items, &D.items);
  for (int i = 0; i < int(H.bvh.size()); i++)
    if (H.bvh[i].count > 0) pk->leaves_host.push_back(i);
  const int32_t* lv = nullptr;
  u |= upload(pk, pk->leaves_host, &lv);
  pk->leaves = const_cast<int32_t*>(lv);
  void* st = nullptr;
  if (cudaMalloc(&st, kStatCount * sizeof(unsigned long long)) == cudaSuccess) {
    pk->owned.push_back(st);
    pk->d_stats = static_cast<unsigned long long*>(st);
  } else {
    u |= ICAM_ERR_CUDA;
  }
  if (u != ICAM_OK || cudaStreamSynchronize(pk->stream) != cudaSuccess) {
    report("upload: " + pk->err);
    icam_pack_destroy(pk);
    return ICAM_ERR_CUDA;
  }
  D.n_faces = int(H.faces.size());
  D.n_subs = int(H.subs.size());
  D.n_edges = int(H.edges.size());
  D.n_pieces = int(H.pieces.size());
  D.n_verts = int(H.verts.size());
  D.n_bvh = int(H.bvh.size());
  D.n_items = int(H.items.size());
  D.tol = H.tol;
  for (int k = 0; k < 3; k++) D.lo[k] = H.lo[k], D.hi[k] = H.hi[k];
  *out = pk;
  return ICAM_OK;
}

void icam_pack_destroy(IcamPack* pk) {
  if (!pk) return;
  cudaSetDevice(pk->device);
  if (pk->stream) cudaStreamSynchronize(pk->stream);
  for (void* p : pk->owned) cudaFree(p);
  for (auto& b : pk->scratch)
    if (b.p) cudaFree(b.p);
  if (pk->stream) cudaStreamDestroy(pk->stream);
  delete pk;
}

int icam_pack_info(const IcamPack* pk, int64_t counts[7]) {
  if (!pk || !counts) return ICAM_ERR_ARG;
  counts[0] = pk->host.faces.size();
  counts[1] = pk->host.edges.size();
  counts[2] = pk->host.verts.size();
  counts[3] = pk->host.subs.size();
  counts[4] = pk->host.pieces.size();
  counts[5] = pk->host.cells.size();
  counts[6] = pk->host.bvh.size();
  return ICAM_OK;
}

const char* icam_last_error(const IcamPack* pk) { return pk ? pk->err.c_str() : "null pack"; }

int icam_pack_box(const IcamPack* pk, double lo[3], double hi[3]) {
  if (!pk || !lo || !hi) return ICAM_ERR_ARG;
  for (int k = 0; k < 3; k++) lo[k] = pk->host.lo[k], hi[k] = pk->host.hi[k];
  return ICAM_OK;
}

void* icam_pack_stream(const IcamPack* pk) { return pk ? static_cast<void*>(pk->stream) : nullptr; }

int icam_points(IcamPack* pk, const double* xyz, size_t n, double clamp, int capped, int precision,
                double* value_out, int8_t* flag_out) {
  if (!pk || (!xyz && n) || (!value_out && n) || (!flag_out && n)) return fail(pk, ICAM_ERR_ARG, "null argument");
  if (precision < ICAM_FP64 || precision > ICAM_MIXED_LEARNED) return fail(pk, ICAM_ERR_ARG, "unknown precision");
  // Scattered points share no centre, so the mixed forms' float solves (seeded and
  // rebased per brick) have nothing to stand on: points are read in double precision only.
  if (precision != ICAM_FP64)
    return fail(pk, ICAM_ERR_ARG, "icam_points reads in ICAM_FP64 only (the mixed forms are brick reads)");
  if (n == 0) return ICAM_OK;
  CK(cudaSetDevice(pk->device));
  void *dx, *dv, *df;
  int r;
  if ((r = scratch(pk, 0, n * 3 * sizeof(double), &dx)) || (r = scratch(pk, 1, n * sizeof(double), &dv)) ||
      (r = scratch(pk, 2, n, &df)))
    return r;
  CK(cudaMemcpyAsync(dx, xyz, n * 3 * sizeof(double), cudaMemcpyHostToDevice, pk->stream));
  double cap = capped ? clamp : INFINITY;
  k_points<<<grid_for(int64_t(n), 128), 128, 0, pk->stream>>>(pk->dev, (const double*)dx, int64_t(n), cap,
                                                               (double*)dv, (int8_t*)df);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(value_out, dv, n * sizeof(double), cudaMemcpyDeviceToHost, pk->stream));
  CK(cudaMemcpyAsync(flag_out, df, n, cudaMemcpyDeviceToHost, pk->stream));
  CK(cudaStreamSynchronize(pk->stream));
  return ICAM_OK;
}

int icam_bricks(IcamPack* pk, const double* first_nodes, size_t n, double h, double clamp, int precision,
                float* values_out, double* d_out) {
  if (!pk || (!first_nodes && n)) return fail(pk, ICAM_ERR_ARG, "null argument");
  if (!(h > 0) || !(clamp > 0)) return fail(pk, ICAM_ERR_ARG, "h and clamp must be positive");
  if (precision < ICAM_FP64 || precision > ICAM_MIXED_LEARNED) return fail(pk, ICAM_ERR_ARG, "unknown precision");
  if (n == 0) return ICAM_OK;
  CK(cudaSetDevice(pk->device));
  void *dfirst, *dval, *dflag;
  int r;
  if ((r = scratch(pk, 0, n * 3 * sizeof(double), &dfirst)) || (r = scratch(pk, 1, n * 729 * sizeof(double), &dval)) ||
      (r = scratch(pk, 2, n * 729, &dflag)))
    return r;
  CK(cudaMemcpyAsync(dfirst, first_nodes, n * 3 * sizeof(double), cudaMemcpyHostToDevice, pk->stream));
  BrickArgs a{};
  a.P = pk->dev;
  a.firsts = (const double*)dfirst;
  a.dcs = nullptr;
  a.n = int64_t(n);
  a.h = h;
  a.clamp = clamp;
  a.leaves = pk->leaves;
  a.n_leaves = int32_t(pk->leaves_host.size());
  a.mixed = precision != ICAM_FP64;
  if ((r = learned_starts(pk, precision, &a))) return r;
  a.d_out = (double*)dval;
  a.flag_out = (int8_t*)dflag;
  a.stats = pk->d_stats;
  CK(cudaMemsetAsync(pk->d_stats, 0, kStatCount * sizeof(unsigned long long), pk->stream));
  launch_bricks(a, pk->stream);
  CK(cudaGetLastError());
  std::vector<double> v(n * 729);
  std::vector<int8_t> f(n * 729);
  unsigned long long st[kStatCount];
  CK(cudaMemcpyAsync(v.data(), dval, n * 729 * sizeof(double), cudaMemcpyDeviceToHost, pk->stream));
  CK(cudaMemcpyAsync(f.data(), dflag, n * 729, cudaMemcpyDeviceToHost, pk->stream));
  CK(cudaMemcpyAsync(st, pk->d_stats, sizeof(st), cudaMemcpyDeviceToHost, pk->stream));
  CK(cudaStreamSynchronize(pk->stream));
  if (st[13]) return fail(pk, ICAM_ERR_BUDGET, "a bulk copy of control nets did not complete in time");
  for (size_t i = 0; i < n * 729; i++) {
    if (values_out) {
      values_out[2 * i] = float(v[i]);
      values_out[2 * i + 1] = float(f[i]);
    }
    if (d_out) d_out[i] = v[i];
  }
  return ICAM_OK;
}

}  // extern "C"

// The level's box decision (partcache.rs:226-331) on the pack's stream, through the
// read bricks sorted in brick order (partcache.rs:486); results in scratch 3, 9, 10.
// The first boxes of a level's decision, on the grid aligned on the origin
// (partcache.rs:250-270); returns their size in bricks.
long long first_boxes(const LevelDesc& L, std::vector<Box4>* out, long long dims[3]) {
  const int64_t* nb = L.nb;
  const double* lo = L.lo;
  const double* origin = L.has_origin ? L.origin : nullptr;
  long long nbmax = std::max(nb[0], std::max(nb[1], nb[2]));
  long long size = 1;
  // The reference starts from one box over the whole level; here from boxes of at most
  // 8 bricks a side. Every box a coarser start would settle is settled the same way by
  // the boxes inside it (grown by the clamp, a child's ball lies in its parent's), so the
  // map is the same, and the coarse boxes, each read within tens of mm, are spared; the
  // first boxes far from the part take their sign from a neighbour (k_first_signs)
  // instead of a reading without a bound. Measured on the freeform part at h = 0.1:
  // one box 56 ms, boxes of 32 bricks 44 ms, boxes of 8 bricks 28 ms.
  while (size < nbmax && size < 8) size *= 2;
  double side = 8.0 * L.h;
  double o[3] = {origin ? origin[0] - L.h : lo[0] - 0.0, origin ? origin[1] - L.h : lo[1], origin ? origin[2] - L.h : lo[2]};
  long long g0[3], start[3];
  for (int k = 0; k < 3; k++) {
    g0[k] = origin ? (long long)std::llround((lo[k] - o[k]) / side) : 0;
    long long q = g0[k] >= 0 ? g0[k] / size : -((-g0[k] + size - 1) / size);
    start[k] = q * size - g0[k];
  }
  out->clear();
  for (long long z = start[2]; z < nb[2]; z += size)
    for (long long y = start[1]; y < nb[1]; y += size)
      for (long long x = start[0]; x < nb[0]; x += size) out->push_back({x, y, z, NAN, INFINITY});
  if (dims)
    for (int k = 0; k < 3; k++) dims[k] = (nb[k] - start[k] + size - 1) / size;
  return size;
}

// The decision's device counters: 0 unused, 1 bricks to read, 2 centres read again in
// double, then one box count a size from kSizeSlot on (at most 4 sizes and their end).
constexpr int kSizeSlot = 4;
constexpr int kCounts = kSizeSlot + 8;

int decide_level(IcamPack* pk, const LevelDesc& L, DecideOut* out) {
  const double h = L.h, clamp = L.clamp;
  const double* lo = L.lo;
  const int64_t* nb = L.nb;
  if (!(h > 0) || !(clamp > 0)) return fail(pk, ICAM_ERR_ARG, "h and clamp must be positive");
  if (nb[0] <= 0 || nb[1] <= 0 || nb[2] <= 0) return fail(pk, ICAM_ERR_ARG, "nb must be positive");
  CK(cudaSetDevice(pk->device));
  cudaStream_t s = pk->stream;
  int64_t total = nb[0] * nb[1] * nb[2];
  if (total > (int64_t(1) << 34)) return fail(pk, ICAM_ERR_ARG, "level too large");
  int64_t launches = 0;
  void *d_map, *d_cur, *d_next, *d_ridx, *d_rdc, *d_cnt;
  int r;
  // box lists: at most 8x the boxes of the previous size; bounded by the level's bricks
  int64_t box_cap = std::max<int64_t>(total + 64, 1 << 12);
  if ((r = scratch(pk, 3, total * sizeof(uint32_t), &d_map)) || (r = scratch(pk, 4, box_cap * sizeof(Box4), &d_cur)) ||
      (r = scratch(pk, 5, box_cap * sizeof(Box4), &d_next)) || (r = scratch(pk, 6, total * sizeof(int64_t), &d_ridx)) ||
      (r = scratch(pk, 7, total * sizeof(double), &d_rdc)) || (r = scratch(pk, 8, kCounts * sizeof(unsigned long long), &d_cnt)))
    return r;
  CK(cudaMemsetAsync(d_cnt, 0, kCounts * sizeof(unsigned long long), s));
  std::vector<Box4> first;
  long long dims[3];
  long long size = first_boxes(L, &first, dims);
  void* d_first;
  if ((r = scratch(pk, 16, first.size() * (sizeof(double) + 1) + 16, &d_first))) return r;
  CK(cudaMemcpyAsync(d_cur, first.data(), first.size() * sizeof(Box4), cudaMemcpyHostToDevice, s));
  out->h2d_bytes = int64_t(first.size() * sizeof(Box4));
  out->d2h_bytes = 0;
  int64_t ncur = int64_t(first.size()), boxes_read = 0;
  unsigned long long* cnt = (unsigned long long*)d_cnt;
  // One launch a box size (size, size / 2, ..., 1), back to back: size k's boxes are the
  // ones size k - 1 appended, counted in slot kSizeSlot + k on the device, which the
  // kernels read themselves (the first size's count is the host's); the host reads the
  // counts back once, after the last size.
  int rounds = 0;
  for (long long s2 = size; s2 >= 1; s2 /= 2) rounds++;
  if (kSizeSlot + rounds + 1 > kCounts) return fail(pk, ICAM_ERR_ARG, "too many box sizes");
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  for (int k = 0; k < rounds; k++) {
    DecideArgs a{};
    a.P = pk->dev;
    a.leaves = pk->leaves;
    a.n_leaves = int32_t(pk->leaves_host.size());
    a.boxes = (const Box4*)(k % 2 == 0 ? d_cur : d_next);
    a.n = k == 0 ? ncur : box_cap;
    a.n_in = k == 0 ? nullptr : cnt + kSizeSlot + k;
    a.sms = sms;
    a.size = size >> k;
    a.h = h;
    a.clamp = clamp;
    for (int q = 0; q < 3; q++) a.lo[q] = lo[q], a.nb[q] = nb[q];
    a.map = (uint32_t*)d_map;
    a.next = (Box4*)(k % 2 == 0 ? d_next : d_cur);
    a.next_cap = box_cap;
    a.n_next = cnt + kSizeSlot + k + 1;
    a.read_idx = (int64_t*)d_ridx;
    a.read_dc = (double*)d_rdc;
    a.read_cap = total;
    a.n_read = cnt + 1;
    a.n_double = cnt + 2;
    a.tight = L.tight ? 1 : 0;
    if (k == 0) {
      a.first_sd = static_cast<double*>(d_first);
      a.first_sign = reinterpret_cast<int8_t*>(static_cast<double*>(d_first) + ncur);
      for (int q = 0; q < 3; q++) a.first_dims[q] = dims[q];
    }
    launch_decide(a, s, k == 0, L.precision != ICAM_FP64);
    launches += k == 0 ? 3 : 1;
    CK(cudaGetLastError());
  }
  unsigned long long cnt_host[kCounts] = {};
  CK(cudaMemcpyAsync(cnt_host, cnt, sizeof(cnt_host), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  out->d2h_bytes += sizeof(cnt_host);
  boxes_read = ncur;
  for (int k = 1; k <= rounds; k++) {
    if (cnt_host[kSizeSlot + k] > (unsigned long long)box_cap) return fail(pk, ICAM_ERR_ROOM, "box list overflow");
    if (k < rounds) boxes_read += int64_t(cnt_host[kSizeSlot + k]);
  }
  const unsigned long long nread = cnt_host[1];
  out->centres_double = int64_t(cnt_host[2]);
  const int64_t R = int64_t(nread);
  // the read bricks in brick order (partcache.rs:486)
  void *d_ridx2, *d_rdc2, *d_tmp;
  size_t tmp_bytes = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, (int64_t*)nullptr, (int64_t*)nullptr, (double*)nullptr,
                                  (double*)nullptr, R, 0, 64, s);
  const size_t Rb = size_t(std::max<int64_t>(R, 1));
  if ((r = scratch(pk, 9, Rb * sizeof(int64_t), &d_ridx2)) || (r = scratch(pk, 10, Rb * sizeof(double), &d_rdc2)) ||
      (r = scratch(pk, 11, tmp_bytes + 16, &d_tmp)))
    return r;
  if (R > 0) {
    CK(cub::DeviceRadixSort::SortPairs(d_tmp, tmp_bytes, (const int64_t*)d_ridx, (int64_t*)d_ridx2,
                                       (const double*)d_rdc, (double*)d_rdc2, R, 0, 64, s));
    launches++;
  }
  out->map = static_cast<uint32_t*>(d_map);
  out->read_idx = static_cast<int64_t*>(d_ridx2);
  out->read_dc = static_cast<double*>(d_rdc2);
  out->n_read = R;
  out->boxes_read = boxes_read;
  out->launches = launches;
  return ICAM_OK;
}

extern "C" {

// The level bake; results left in device scratch.
static int bake_level(IcamPack* pk, double h, const double lo[3], const int64_t nb[3], double clamp,
                      const double origin[3], int precision, size_t* n_slots, IcamBakeStats* stats,
                      const uint32_t** d_map_out, const uint32_t** d_atlas_out) {
  if (!pk || !lo || !nb || !n_slots) return fail(pk, ICAM_ERR_ARG, "null argument");
  if (precision < ICAM_FP64 || precision > ICAM_MIXED_LEARNED) return fail(pk, ICAM_ERR_ARG, "unknown precision");
  CK(cudaSetDevice(pk->device));
  cudaStream_t s = pk->stream;
  pk->last_map = pk->last_atlas = nullptr;  // the scratch they live in is about to change
  pk->last_map_entries = pk->last_slots = 0;
  LevelDesc L;
  L.h = h, L.clamp = clamp;
  for (int k = 0; k < 3; k++) L.lo[k] = lo[k], L.nb[k] = nb[k], L.origin[k] = origin ? origin[k] : 0.0;
  L.has_origin = origin != nullptr;
  L.precision = precision;
  L.tight = true;  // a bake: the map and words of the reference's rule with fewer reads
  cudaEvent_t ev[5];
  for (auto& e : ev) CK(cudaEventCreate(&e));
  CK(cudaEventRecord(ev[0], s));
  DecideOut D;
  int r = decide_level(pk, L, &D);
  if (r) {
    for (auto& e : ev) cudaEventDestroy(e);
    return r;
  }
  CK(cudaEventRecord(ev[1], s));
  const int64_t R = D.n_read, boxes_read = D.boxes_read;
  int64_t launches = D.launches;
  void* d_map = D.map;
  void *d_tmp, *d_first, *d_words, *d_kind, *d_flag, *d_slot, *d_atlas;
  size_t tmp_bytes = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, (int64_t*)nullptr, (int64_t*)nullptr, R + 1, s);
  const size_t Rb = size_t(std::max<int64_t>(R, 1));
  if ((r = scratch(pk, 11, tmp_bytes + 16, &d_tmp)) || (r = scratch(pk, 12, Rb * 3 * sizeof(double), &d_first)) ||
      (r = scratch(pk, 13, Rb * WORD_STRIDE * sizeof(uint32_t), &d_words)) || (r = scratch(pk, 14, Rb * sizeof(int32_t), &d_kind)) ||
      (r = scratch(pk, 15, (Rb + 1) * 2 * sizeof(int64_t), &d_flag)))
    return r;
  d_slot = (int64_t*)d_flag + (Rb + 1);
  void* d_ridx2 = D.read_idx;
  void* d_rdc2 = D.read_dc;
  size_t nwords_slots = 0;
  if (R > 0) {
    k_gather_firsts<<<grid_for(R, 256), 256, 0, s>>>((const int64_t*)d_ridx2, R, nb[0], nb[1], h, lo[0], lo[1], lo[2],
                                                    (double*)d_first);
    launches++;
    CK(cudaEventRecord(ev[2], s));
    BrickArgs b{};
    b.P = pk->dev;
    b.firsts = (const double*)d_first;
    b.dcs = (const double*)d_rdc2;
    b.n = R;
    b.h = h;
    b.clamp = clamp;
    b.leaves = pk->leaves;
    b.n_leaves = int32_t(pk->leaves_host.size());
    b.mixed = precision != ICAM_FP64;
    b.kind_only = 1;
    if ((r = learned_starts(pk, precision, &b))) return r;
    b.words_out = (uint32_t*)d_words;
    b.kind_out = (int32_t*)d_kind;
    b.stats = pk->d_stats;
    CK(cudaMemsetAsync(pk->d_stats, 0, kStatCount * sizeof(unsigned long long), s));
    launch_bricks(b, s);
    launches++;
    CK(cudaGetLastError());
    CK(cudaEventRecord(ev[3], s));
    // slots: stored bricks numbered in brick order
    k_is_words<<<grid_for(R, 256), 256, 0, s>>>((const int32_t*)d_kind, R, (int64_t*)d_flag);
    CK(cudaMemsetAsync((int64_t*)d_flag + R, 0, sizeof(int64_t), s));
    CK(cub::DeviceScan::ExclusiveSum(d_tmp, tmp_bytes, (const int64_t*)d_flag, (int64_t*)d_slot, R + 1, s));
    int64_t ns = 0;
    CK(cudaMemcpyAsync(&ns, (int64_t*)d_slot + R, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    D.d2h_bytes += sizeof(ns);
    nwords_slots = size_t(ns);
    if ((r = scratch(pk, 17, std::max<size_t>(nwords_slots, 1) * 365 * sizeof(uint32_t), &d_atlas))) return r;
    k_assemble<<<grid_for(R, 1), 128, 0, s>>>((const int64_t*)d_ridx2, (const int32_t*)d_kind, (const int64_t*)d_slot,
                                              R, (const uint32_t*)d_words, (uint32_t*)d_map, (uint32_t*)d_atlas);
    launches += 3;
    CK(cudaGetLastError());
  } else {
    CK(cudaEventRecord(ev[2], s));
    CK(cudaEventRecord(ev[3], s));
    if ((r = scratch(pk, 17, 365 * sizeof(uint32_t), &d_atlas))) return r;
  }
  CK(cudaEventRecord(ev[4], s));
  CK(cudaStreamSynchronize(s));
  *n_slots = nwords_slots;
  *d_map_out = (const uint32_t*)d_map;
  *d_atlas_out = (const uint32_t*)d_atlas;
  pk->last_map = (const uint32_t*)d_map;
  pk->last_atlas = (const uint32_t*)d_atlas;
  pk->last_map_entries = size_t(nb[0] * nb[1] * nb[2]);
  pk->last_slots = nwords_slots;
  unsigned long long st[kStatCount] = {0};
  if (R > 0) CK(cudaMemcpy(st, pk->d_stats, sizeof(st), cudaMemcpyDeviceToHost));
  if (st[13]) {
    for (auto& e : ev) cudaEventDestroy(e);
    return fail(pk, ICAM_ERR_BUDGET, "a bulk copy of control nets did not complete in time");
  }
  if (stats) {
    std::memset(stats, 0, sizeof(*stats));
    stats->boxes_read = boxes_read;
    stats->bricks_read = R;
    stats->bricks_words = int64_t(nwords_slots);
    stats->nodes_exact = R ? int64_t(st[0]) : 0;
    stats->nodes_far = R ? int64_t(st[1]) : 0;
    stats->nodes_undecided = R ? int64_t(st[2]) : 0;
    stats->pairs = R ? int64_t(st[4]) : 0;
    for (int k = 0; k < 5; k++) stats->census[k] = R ? int64_t(st[6 + k]) : 0;
    stats->bricks_settled = R ? int64_t(st[11]) : 0;
    stats->kernel_launches = launches;
    stats->nodes_double = R ? int64_t(st[12]) : 0;
    stats->centres_double = D.centres_double;
    stats->newton_solves = R ? int64_t(st[17]) : 0;
    stats->newton_evals = R ? int64_t(st[16]) : 0;
    stats->h2d_bytes = D.h2d_bytes;
    stats->d2h_bytes = D.d2h_bytes + int64_t(sizeof(st));
    float ms;
    cudaEventElapsedTime(&ms, ev[0], ev[1]);
    stats->ms_decide = ms;
    cudaEventElapsedTime(&ms, ev[2], ev[3]);
    stats->ms_nodes = ms;
    cudaEventElapsedTime(&ms, ev[3], ev[4]);
    stats->ms_post = ms;
  }
  for (auto& e : ev) cudaEventDestroy(e);
  return ICAM_OK;
}

int icam_bake_level(IcamPack* pk, double h, const double lo[3], const int64_t nb[3], double clamp,
                    const double origin[3], int precision, uint32_t* map_out, uint32_t* atlas_out,
                    size_t atlas_cap_words, size_t* n_slots, IcamBakeStats* stats) {
  const uint32_t *dm, *da;
  int rc = bake_level(pk, h, lo, nb, clamp, origin, precision, n_slots, stats, &dm, &da);
  if (rc) return rc;
  int64_t total = nb[0] * nb[1] * nb[2];
  if (map_out) {
    CK(cudaMemcpyAsync(map_out, dm, total * sizeof(uint32_t), cudaMemcpyDeviceToHost, pk->stream));
    if (stats) stats->d2h_bytes += total * int64_t(sizeof(uint32_t));
  }
  if (atlas_out) {
    if (*n_slots * 365 > atlas_cap_words) return fail(pk, ICAM_ERR_ARG, "atlas_out too small");
    CK(cudaMemcpyAsync(atlas_out, da, *n_slots * 365 * sizeof(uint32_t), cudaMemcpyDeviceToHost, pk->stream));
    if (stats) stats->d2h_bytes += int64_t(*n_slots * 365 * sizeof(uint32_t));
  }
  CK(cudaStreamSynchronize(pk->stream));
  return ICAM_OK;
}

int icam_decide_level(IcamPack* pk, double h, const double lo[3], const int64_t nb[3], double clamp,
                      const double origin[3], int precision, uint32_t* map_out, int64_t* read_out, double* dc_out,
                      size_t read_cap, size_t* n_read, IcamBakeStats* stats) {
  if (!pk || !lo || !nb || !n_read) return fail(pk, ICAM_ERR_ARG, "null argument");
  if (precision < ICAM_FP64 || precision > ICAM_MIXED_LEARNED) return fail(pk, ICAM_ERR_ARG, "unknown precision");
  CK(cudaSetDevice(pk->device));
  cudaStream_t s = pk->stream;
  pk->last_map = pk->last_atlas = nullptr;  // the decision reuses the bake's scratch
  pk->last_map_entries = pk->last_slots = 0;
  LevelDesc L;
  L.h = h, L.clamp = clamp;
  for (int k = 0; k < 3; k++) L.lo[k] = lo[k], L.nb[k] = nb[k], L.origin[k] = origin ? origin[k] : 0.0;
  L.has_origin = origin != nullptr;
  L.precision = precision;
  cudaEvent_t ev[2];
  for (auto& e : ev) CK(cudaEventCreate(&e));
  CK(cudaEventRecord(ev[0], s));
  DecideOut D;
  int r = decide_level(pk, L, &D);
  if (r) {
    for (auto& e : ev) cudaEventDestroy(e);
    return r;
  }
  CK(cudaEventRecord(ev[1], s));
  *n_read = size_t(D.n_read);
  const int64_t total = nb[0] * nb[1] * nb[2];
  if (map_out) CK(cudaMemcpyAsync(map_out, D.map, total * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  const size_t m = std::min(size_t(D.n_read), read_cap);
  if (read_out && m) CK(cudaMemcpyAsync(read_out, D.read_idx, m * sizeof(int64_t), cudaMemcpyDeviceToHost, s));
  if (dc_out && m) CK(cudaMemcpyAsync(dc_out, D.read_dc, m * sizeof(double), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  if (stats) {
    std::memset(stats, 0, sizeof(*stats));
    stats->boxes_read = D.boxes_read;
    stats->bricks_read = D.n_read;
    stats->kernel_launches = D.launches;
    stats->centres_double = D.centres_double;
    stats->h2d_bytes = D.h2d_bytes;
    stats->d2h_bytes = D.d2h_bytes;
    float ms;
    cudaEventElapsedTime(&ms, ev[0], ev[1]);
    stats->ms_decide = ms;
  }
  for (auto& e : ev) cudaEventDestroy(e);
  if ((read_out || dc_out) && size_t(D.n_read) > read_cap)
    return fail(pk, ICAM_ERR_ARG, "icam_decide_level: read_cap is below the bricks to read (*n_read)");
  return ICAM_OK;
}

int icam_level_read(IcamPack* pk, uint32_t* map_out, size_t map_entries, uint32_t* atlas_out,
                    size_t atlas_cap_words) {
  if (!pk) return ICAM_ERR_ARG;
  if (!pk->last_map) return fail(pk, ICAM_ERR_ARG, "icam_level_read: no level baked on this pack");
  if (map_out && map_entries != pk->last_map_entries)
    return fail(pk, ICAM_ERR_ARG, "icam_level_read: map_entries is not the level's brick count");
  if (atlas_out && atlas_cap_words < pk->last_slots * 365)
    return fail(pk, ICAM_ERR_ARG, "icam_level_read: atlas_out holds fewer than n_slots x 365 words");
  CK(cudaSetDevice(pk->device));
  // the direction inferred from the addresses (unified addressing): host arrays, or
  // device memory of this GPU or a peer (a caller that keeps the level on the device)
  if (map_out)
    CK(cudaMemcpyAsync(map_out, pk->last_map, map_entries * sizeof(uint32_t), cudaMemcpyDefault, pk->stream));
  if (atlas_out && pk->last_slots)
    CK(cudaMemcpyAsync(atlas_out, pk->last_atlas, pk->last_slots * 365 * sizeof(uint32_t), cudaMemcpyDefault,
                       pk->stream));
  CK(cudaStreamSynchronize(pk->stream));
  return ICAM_OK;
}

int icam_bake_level_device(IcamPack* pk, double h, const double lo[3], const int64_t nb[3], double clamp,
                           const double origin[3], int precision, const uint32_t** d_map, const uint32_t** d_atlas,
                           size_t* n_slots, IcamBakeStats* stats) {
  if (!d_map || !d_atlas) return fail(pk, ICAM_ERR_ARG, "null argument");
  return bake_level(pk, h, lo, nb, clamp, origin, precision, n_slots, stats, d_map, d_atlas);
}

int icam_list(const IcamPack* pk, const double c[3], double r, double d, uint32_t* codes, size_t cap, size_t* n) {
  if (!pk || !c || !n) return ICAM_ERR_ARG;
  const HostPack& H = pk->host;
  double reach = d + 2.0 * r;
  V cc(c[0], c[1], c[2]);
  size_t k = 0;
  std::vector<int> stack = {0};
  while (!stack.empty()) {
    const DBvh& nd = H.bvh[stack.back()];
    stack.pop_back();
    Bx b;
    b.add(V(nd.lo[0], nd.lo[1], nd.lo[2]));
    b.add(V(nd.hi[0], nd.hi[1], nd.hi[2]));
    if (b.dist(cc) > reach) continue;
    if (nd.count == 0) {
      stack.push_back(nd.first);
      stack.push_back(nd.first + 1);
      continue;
    }
    for (int i = 0; i < nd.count; i++) {
      uint32_t code = H.items[nd.first + i];
      uint32_t kind = code >> IK_SHIFT, idx = code & IK_MASK;
      const double* box = kind == IK_FACE ? H.faces[idx].box
                          : kind == IK_SUB ? H.subs[idx].box
                          : kind == IK_EDGE ? H.edges[idx].box
                          : kind == IK_PIECE ? H.pieces[idx].box
                                             : nullptr;
      double lb;
      if (box) {
        Bx ib;
        ib.add(V(box[0], box[1], box[2]));
        ib.add(V(box[3], box[4], box[5]));
        lb = ib.dist(cc);
      } else {
        lb = (cc - V(H.verts[idx].p[0], H.verts[idx].p[1], H.verts[idx].p[2])).len();
      }
      if (lb <= reach) {
        if (k < cap && codes) codes[k] = code;
        k++;
      }
    }
  }
  *n = k;
  return ICAM_OK;
}

int icam_probe_fma(IcamPack* pk, int precision, double* flops) {
  if (!pk || !flops) return ICAM_ERR_ARG;
  CK(cudaSetDevice(pk->device));
  int sms = 0;
  CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, pk->device));
  void* d;
  int r;
  if ((r = scratch(pk, 0, 64, &d))) return r;
  const int blocks = sms * 8, threads = 256, iters = 1 << 14;
  cudaEvent_t a, b;
  CK(cudaEventCreate(&a));
  CK(cudaEventCreate(&b));
  float best = 1e30f;
  for (int rep = 0; rep < 5; rep++) {
    CK(cudaEventRecord(a, pk->stream));
    launch_fma(precision == ICAM_FP64, d, blocks, threads, iters, pk->stream);
    CK(cudaEventRecord(b, pk->stream));
    CK(cudaEventSynchronize(b));
    float ms;
    CK(cudaEventElapsedTime(&ms, a, b));
    if (rep > 0) best = std::min(best, ms);
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  *flops = 2.0 * 8.0 * double(iters) * blocks * threads / (best * 1e-3);
  return ICAM_OK;
}

int icam_warm(IcamPack* pk, double secs) {
  if (!pk) return ICAM_ERR_ARG;
  CK(cudaSetDevice(pk->device));
  void* d;
  int r;
  if ((r = scratch(pk, 0, 64, &d))) return r;
  auto t0 = std::chrono::steady_clock::now();
  while (std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() < secs) {
    k_warm<<<1024, 256, 0, pk->stream>>>((float*)d, 4096);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(pk->stream));
  }
  return ICAM_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// The brick read without allocation (icam_bricks_static).
//
// icam_bricks grows the pack's scratch buffers with cudaMalloc / cudaFree when a
// call asks for more bricks than any call before it, and converts the values in a
// host std::vector. Some callers cannot have either: a machining simulation that
// has reserved the GPU's memory for its stock model up front leaves nothing for the
// library to take, and a control loop that reads bricks between its own
// stream-ordered kernels cannot afford cudaFree, which waits for the whole device to
// go idle. This variant runs the same brick kernel with every buffer it needs
// (first nodes, node values and flags, the float pairs, the kernel's counters) in one
// file-scope device array of fixed size, so a call allocates nothing, on the device
// or on the host. The array holds at most ICAM_STATIC_BRICKS bricks (about 3 MB);
// larger requests are refused, and the caller splits them.
//
// The array is one per device and every call on that device shares it: two calls
// that overlap in time (from two threads, or on two packs of one device) race on it
// and must be serialised by the caller. The kernel's counters are the only part that
// must start at zero; each call clears them on the pack's stream before the kernel.
// The first call on a device looks the array's address up (cudaGetSymbolAddress,
// with that device current), which may load this library's device code; make that
// first call before any stream capture. The address is kept for the life of the
// process: after a cudaDeviceReset of that device (which unloads the array) it is
// stale, so no call may follow a reset.
// ---------------------------------------------------------------------------

namespace {

constexpr size_t kStaticStats = 0;  // the brick kernel's kStatCount counters
constexpr size_t kStaticFirst = 256;
constexpr size_t kStaticD = kStaticFirst + size_t(ICAM_STATIC_BRICKS) * 3 * sizeof(double);
constexpr size_t kStaticPairs = kStaticD + size_t(ICAM_STATIC_BRICKS) * ICAM_NODES * sizeof(double);
constexpr size_t kStaticFlag = kStaticPairs + size_t(ICAM_STATIC_BRICKS) * ICAM_NODES * 2 * sizeof(float);
constexpr size_t kStaticBytes = kStaticFlag + size_t(ICAM_STATIC_BRICKS) * ICAM_NODES;
static_assert(kStatCount * sizeof(unsigned long long) <= kStaticFirst, "the counters fit before the first nodes");
static_assert(kStaticFirst % 256 == 0 && kStaticD % 256 == 0 && kStaticPairs % 256 == 0 && kStaticFlag % 256 == 0,
              "static scratch regions are 256-byte aligned");

constexpr int kStaticDevices = 64;
std::atomic<void*> g_static_addr[kStaticDevices];

// (value, flag) float pairs from the double values and the flags, converted as
// icam_bricks converts them on the host.
__global__ void k_static_pairs(const double* d, const int8_t* f, int64_t m, float2* pairs) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < m; i += int64_t(gridDim.x) * blockDim.x)
    pairs[i] = make_float2(float(d[i]), float(f[i]));
}

int static_fail(char* err, size_t errlen, int code, const char* what, const char* detail) {
  if (err && errlen) std::snprintf(err, errlen, "icam_bricks_static: %s%s%s", what, detail ? ": " : "", detail ? detail : "");
  return code;
}

}  // namespace

static __device__ __align__(256) unsigned char g_static_scratch[kStaticBytes];

#define SCK(call)                                                                                \
  do {                                                                                           \
    cudaError_t e_ = (call);                                                                     \
    if (e_ != cudaSuccess) return static_fail(err, errlen, ICAM_ERR_CUDA, #call, cudaGetErrorString(e_)); \
  } while (0)

extern "C" int icam_bricks_static(IcamPack* pk, const double* first_nodes, size_t n, double h, double clamp,
                                  int precision, float* values_out, double* d_out, char* err, size_t errlen) {
  if (!pk || (!first_nodes && n)) return static_fail(err, errlen, ICAM_ERR_ARG, "null argument", nullptr);
  if (!(h > 0) || !(clamp > 0)) return static_fail(err, errlen, ICAM_ERR_ARG, "h and clamp must be positive", nullptr);
  if (precision < ICAM_FP64 || precision > ICAM_MIXED_LEARNED)
    return static_fail(err, errlen, ICAM_ERR_ARG, "unknown precision", nullptr);
  if (n > size_t(ICAM_STATIC_BRICKS)) {
    char detail[96];
    std::snprintf(detail, sizeof detail, "%zu bricks asked, at most %d per call", n, ICAM_STATIC_BRICKS);
    return static_fail(err, errlen, ICAM_ERR_ROOM, "more bricks than the static scratch holds", detail);
  }
  if (pk->device < 0 || pk->device >= kStaticDevices)
    return static_fail(err, errlen, ICAM_ERR_ARG, "device ordinal out of range", nullptr);
  // ICAM_MIXED_LEARNED needs the pack's trained seed network, as icam_bricks does
  if (precision == ICAM_MIXED_LEARNED && !pk->net.ready && pk->dev.n_subs > 0)
    return static_fail(err, errlen, ICAM_ERR_ARG,
                       "ICAM_MIXED_LEARNED: train (icam_seednet_train) or load the seed network first", nullptr);
  if (n == 0) return ICAM_OK;
  SCK(cudaSetDevice(pk->device));
  unsigned char* base = static_cast<unsigned char*>(g_static_addr[pk->device].load(std::memory_order_acquire));
  if (!base) {
    void* p = nullptr;
    SCK(cudaGetSymbolAddress(&p, g_static_scratch));
    g_static_addr[pk->device].store(p, std::memory_order_release);
    base = static_cast<unsigned char*>(p);
  }
  auto* stats = reinterpret_cast<unsigned long long*>(base + kStaticStats);
  auto* dfirst = reinterpret_cast<double*>(base + kStaticFirst);
  auto* dval = reinterpret_cast<double*>(base + kStaticD);
  auto* dpairs = reinterpret_cast<float2*>(base + kStaticPairs);
  auto* dflag = reinterpret_cast<int8_t*>(base + kStaticFlag);
  const int64_t m = int64_t(n) * ICAM_NODES;
  SCK(cudaMemcpyAsync(dfirst, first_nodes, n * 3 * sizeof(double), cudaMemcpyHostToDevice, pk->stream));
  SCK(cudaMemsetAsync(stats, 0, kStatCount * sizeof(unsigned long long), pk->stream));
  BrickArgs a{};
  a.P = pk->dev;
  a.firsts = dfirst;
  a.dcs = nullptr;
  a.n = int64_t(n);
  a.h = h;
  a.clamp = clamp;
  a.leaves = pk->leaves;
  a.n_leaves = int32_t(pk->leaves_host.size());
  a.mixed = precision != ICAM_FP64;
  if (precision == ICAM_MIXED_LEARNED && pk->dev.n_subs > 0) {  // the seed network's starts, as icam_bricks takes them
    a.net_feat = pk->net.feat;
    a.net_w = pk->net.wbf;
  }
  a.d_out = dval;
  a.flag_out = dflag;
  a.stats = stats;
  launch_bricks(a, pk->stream);
  SCK(cudaGetLastError());
  if (values_out) {
    k_static_pairs<<<grid_for(m, 256), 256, 0, pk->stream>>>(dval, dflag, m, dpairs);
    SCK(cudaGetLastError());
    SCK(cudaMemcpyAsync(values_out, dpairs, size_t(m) * sizeof(float2), cudaMemcpyDeviceToHost, pk->stream));
  }
  if (d_out) SCK(cudaMemcpyAsync(d_out, dval, size_t(m) * sizeof(double), cudaMemcpyDeviceToHost, pk->stream));
  SCK(cudaStreamSynchronize(pk->stream));
  return ICAM_OK;
}

#undef SCK
