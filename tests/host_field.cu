// Test infrastructure: the library's double-precision point query (field.cuh, whose
// functions are __host__ __device__) built for the host, so that CPU tests run the same
// search as the k_points kernel over a pack made by the same builder. Not part of the
// library.
#include <cstdio>
#include <string>

#include "../implicitcam_b200/csrc/field.cuh"
#include "../implicitcam_b200/csrc/pack_build.h"

using namespace icam;

// Packs the solid (need as the library's default) and answers each point as k_points
// does: value and flag (0 exact, 1 past the cap, 2 undecided). Returns 0, or 1 with the
// pack's message in err.
extern "C" int host_points(const IcamSolidDesc* d, double need, const double* xyz, long n, double cap,
                           double* value, int* flag, char* err, size_t errlen) {
  HostPack H;
  std::string msg;
  if (!build_pack(d, need, &H, &msg)) {
    if (err && errlen) snprintf(err, errlen, "%s", msg.c_str());
    return 1;
  }
  DPack D{};
  D.faces = H.faces.data();
  D.nurbs = H.nurbs.data();
  D.subs = H.subs.data();
  D.sub_cp = H.sub_cp.data();
  D.sub_cp32 = H.sub_cp32.data();
  D.span_cp = H.span_cp.data();
  D.breaks = H.breaks.data();
  D.edges = H.edges.data();
  D.pieces = H.pieces.data();
  D.verts = H.verts.data();
  D.cells = H.cells.data();
  D.insts = H.insts.data();
  D.among = H.among.data();
  D.tpieces = H.tpieces.data();
  D.bvh = H.bvh.data();
  D.items = H.items.data();
  D.n_faces = int32_t(H.faces.size());
  D.n_subs = int32_t(H.subs.size());
  D.n_edges = int32_t(H.edges.size());
  D.n_pieces = int32_t(H.pieces.size());
  D.n_verts = int32_t(H.verts.size());
  D.n_bvh = int32_t(H.bvh.size());
  D.n_items = int32_t(H.items.size());
  D.tol = H.tol;
  for (int k = 0; k < 3; k++) D.lo[k] = H.lo[k], D.hi[k] = H.hi[k];
  for (long i = 0; i < n; i++) {
    Acc A;
    point_query(D, make_double3(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]), cap, A);
    double v;
    int f;
    finish(A, cap, &v, &f);
    value[i] = v;
    flag[i] = f;
  }
  return 0;
}
