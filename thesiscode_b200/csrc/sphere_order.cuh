// Spatially coherent order of points on (or near) the unit sphere: a 31-bit
// key = cube face (its rank, 3 bits) and the index along a 2-D Hilbert curve
// over that face (14 bits per axis). The point is projected from the origin onto the
// face of its largest |coordinate| (gnomonic projection), so consecutive keys
// are consecutive cells of a 2-D curve on the surface: runs of a few hundred
// keys form compact patches, unlike a 3-D curve through the cube, whose runs
// cut the spherical shell into elongated or split pieces (on the level-7
// icosahedral grid a run of 384 points had a median radius 2.4x that of a
// disk of the same area under a 10-bit 3-D Hilbert curve, 1.6x here).
//
// The faces are visited in the order +x, +y, -x, -z, -y, +z, each with its
// (u, v) axes swapped or reflected so that the curve on one face ends at the
// cube corner where the curve on the next face starts: the whole curve is
// continuous, and a run of keys that crosses from one face to the next stays
// a compact patch around the shared corner (with faces in plain index order
// such runs joined two distant regions: level-6 runs of 384 points reached a
// radius of 1.6 rad, 0.31 rad with the continuous order). The order and
// orientations were found by a search over the 6 faces x 8 orientations for
// chains whose end and start corners coincide.
//
// 2-D Hilbert index: the published rotate-and-reflect construction
// (coordinates to distance, most significant quadrant first; e.g. H. S.
// Warren, "Hacker's Delight", 2nd ed., ch. 16).
#pragma once
#include <cuda_runtime.h>

namespace tcb {

constexpr int kFaceBits = 14;  // cells per face axis: 16384 (about 1.2e-4 rad)
constexpr int kSphereKeyBits = 3 + 2 * kFaceBits;
// face f = 2*axis + (coordinate < 0): its rank along the curve (3 bits per
// face) and whether its (u, v) are swapped, u reflected, v reflected (bit f)
constexpr unsigned kFaceRank = 0x1d850u;
constexpr unsigned kFaceSwap = 0x08u, kFaceFlipU = 0x16u, kFaceFlipV = 0x08u;

__device__ __forceinline__ unsigned sphere_key(double x, double y, double z) {
  const double ax = fabs(x), ay = fabs(y), az = fabs(z);
  int axis;
  double major, u, v;
  if (ax >= ay && ax >= az) {
    axis = 0;
    major = x;
    u = y;
    v = z;
  } else if (ay >= az) {
    axis = 1;
    major = y;
    u = x;
    v = z;
  } else {
    axis = 2;
    major = z;
    u = x;
    v = y;
  }
  const unsigned face = 2u * (unsigned)axis + (major < 0.0 ? 1u : 0u);
  if ((kFaceSwap >> face) & 1u) {
    const double t = u;
    u = v;
    v = t;
  }
  if ((kFaceFlipU >> face) & 1u) u = -u;
  if ((kFaceFlipV >> face) & 1u) v = -v;
  const double inv = major != 0.0 ? 1.0 / fabs(major) : 0.0;
  const int n = 1 << kFaceBits;
  double qu = (u * inv + 1.0) * 0.5 * n, qv = (v * inv + 1.0) * 0.5 * n;
  // fmax/fmin also send a NaN coordinate (a non-finite input) to cell 0
  qu = fmin(fmax(qu, 0.0), (double)(n - 1));
  qv = fmin(fmax(qv, 0.0), (double)(n - 1));
  unsigned X = (unsigned)qu, Y = (unsigned)qv, d = 0;
  for (unsigned s = (unsigned)n >> 1; s > 0; s >>= 1) {
    const unsigned rx = (X & s) ? 1u : 0u, ry = (Y & s) ? 1u : 0u;
    d += s * s * ((3u * rx) ^ ry);
    if (ry == 0) {  // rotate the quadrant
      if (rx == 1) {
        X = (unsigned)n - 1 - X;
        Y = (unsigned)n - 1 - Y;
      }
      const unsigned t = X;
      X = Y;
      Y = t;
    }
  }
  return (((kFaceRank >> (3u * face)) & 7u) << (2 * kFaceBits)) | d;
}

}  // namespace tcb
