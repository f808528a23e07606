// Mask construction of the 3D step on the device: Aerolume ns3d/geometry.py:385-495
// (build_geometry3d) with its exact signed distance to the bodies' triangle meshes
// (geometry.py:68-196 mesh_signed_distance, 229-262 grid_signed_distance without the shared
// voxeliser).
//
// Per body and staggered grid (u, v, w faces and cells of the body window), one thread per
// grid point scans all triangles of the body, staged in shared memory 256 at a time: the
// nearest triangle (first index of the smallest squared distance; a triangle whose bounding
// ball lies farther than the nearest distance so far is skipped, which cannot change the
// selection) and the generalised winding number (sum of signed solid angles over every
// triangle; inside when its magnitude exceeds 1/2).  Each
// point nearest to a face's interior and off its plane votes for the face's outward side
// (integer atomics, so the tally is exact); a second pass gives a point within the plane
// zone of its face that face's signed plane distance with the voted side (else the mesh's
// orientation), every other point the winding sign times its distance.  The assembly kernel
// turns the per-body distances of one grid into the smooth solid fraction with the boundary
// faces zeroed, the combined mask, the rigid-spin solid velocity and the per-body force and
// moment weights.  Arithmetic follows the reference operation by operation in the working
// precision.
#include <cstdint>
#include <limits>

#include "host_common.cuh"

namespace aero {
namespace masks {

constexpr int NT = 256;   // threads per block
constexpr int TCH = 256;  // triangles per shared-memory chunk

template <typename T>
struct Tri {
  T ax, ay, az, bx, by, bz, cx, cy, cz;
  T mx, my, mz, rad;  // a ball holding the triangle: its centroid and the largest vertex distance
};

// squared distance of p to the triangle (geometry.py:68-109)
template <typename T>
__device__ __forceinline__ T tri_d2(T px, T py, T pz, const Tri<T> &t) {
  const T tiny = std::numeric_limits<T>::min();
  const T e0x = t.bx - t.ax, e0y = t.by - t.ay, e0z = t.bz - t.az;
  const T e1x = t.cx - t.bx, e1y = t.cy - t.by, e1z = t.cz - t.bz;
  const T e2x = t.ax - t.cx, e2y = t.ay - t.cy, e2z = t.az - t.cz;
  const T nx = e0y * (-e2z) - e0z * (-e2y);
  const T ny = e0z * (-e2x) - e0x * (-e2z);
  const T nz = e0x * (-e2y) - e0y * (-e2x);
  const T nn = (nx * nx + ny * ny) + nz * nz;
  const T w0x = px - t.ax, w0y = py - t.ay, w0z = pz - t.az;
  const T w1x = px - t.bx, w1y = py - t.by, w1z = pz - t.bz;
  const T w2x = px - t.cx, w2y = py - t.cy, w2z = pz - t.cz;
  auto side = [&](T ex, T ey, T ez, T wx, T wy, T wz) {
    const T cxp = ey * wz - ez * wy, cyp = ez * wx - ex * wz, czp = ex * wy - ey * wx;
    return (nx * cxp + ny * cyp) + nz * czp;
  };
  const bool inside = side(e0x, e0y, e0z, w0x, w0y, w0z) >= T(0) && side(e1x, e1y, e1z, w1x, w1y, w1z) >= T(0) &&
                      side(e2x, e2y, e2z, w2x, w2y, w2z) >= T(0) && nn > tiny;
  if (inside) {
    const T pd = (nx * w0x + ny * w0y) + nz * w0z;
    return pd * pd / (nn > tiny ? nn : tiny);
  }
  auto seg = [&](T ex, T ey, T ez, T wx, T wy, T wz) {
    T ee = (ex * ex + ey * ey) + ez * ez;
    ee = ee > tiny ? ee : tiny;
    T s = ((wx * ex + wy * ey) + wz * ez) / ee;
    s = s > T(0) ? (s < T(1) ? s : T(1)) : T(0);
    const T dx = wx - s * ex, dy = wy - s * ey, dz = wz - s * ez;
    return (dx * dx + dy * dy) + dz * dz;
  };
  const T s0 = seg(e0x, e0y, e0z, w0x, w0y, w0z);
  const T s1 = seg(e1x, e1y, e1z, w1x, w1y, w1z);
  const T s2 = seg(e2x, e2y, e2z, w2x, w2y, w2z);
  const T m = s1 < s0 ? s1 : s0;
  return s2 < m ? s2 : m;
}

// signed solid angle of the triangle seen from p (geometry.py:112-123, van Oosterom and
// Strackee 1983)
template <typename T>
__device__ __forceinline__ T solid_angle(T px, T py, T pz, const Tri<T> &t) {
  const T ax = t.ax - px, ay = t.ay - py, az = t.az - pz;
  const T bx = t.bx - px, by = t.by - py, bz = t.bz - pz;
  const T cx = t.cx - px, cy = t.cy - py, cz = t.cz - pz;
  const T la = sqrt((ax * ax + ay * ay) + az * az);
  const T lb = sqrt((bx * bx + by * by) + bz * bz);
  const T lc = sqrt((cx * cx + cy * cy) + cz * cz);
  const T det = (ax * (by * cz - bz * cy) + ay * (bz * cx - bx * cz)) + az * (bx * cy - by * cx);
  const T den = (((la * lb) * lc + ((ax * bx + ay * by) + az * bz) * lc) + ((bx * cx + by * cy) + bz * cz) * la) +
                ((cx * ax + cy * ay) + cz * az) * lb;
  return T(2) * atan2(det, den);
}

template <typename T>
struct SdfParams {
  const T *verts;
  int nvert;
  const int32_t *faces;
  int nface;
  const T *pts;              // (npt, 3), or NULL: the centres of the grid below
  long long npt;
  int gnx, gny;              // grid: x fastest, then y, then z
  T gx, gy, gz, h;           // origins of the first centre minus h / 2, cell size
  T zone;                    // plane zone
  int *best;                 // (npt) nearest triangle
  unsigned char *flag;       // (npt) bit 0 inside, bit 1 in the plane of the nearest face
  T *dist, *dpl;             // (npt) distance to the nearest triangle, signed plane distance
  int *votes;                // (nface) outward-side tally
  const int *orient;         // the mesh's orientation sign
  T *out;                    // (npt) signed distance
};

template <typename T>
__device__ __forceinline__ void point_of(const SdfParams<T> &P, long long q, T &px, T &py, T &pz) {
  if (P.pts) {
    px = P.pts[3 * q];
    py = P.pts[3 * q + 1];
    pz = P.pts[3 * q + 2];
    return;
  }
  const long long plane = (long long)P.gnx * P.gny;
  const int k = (int)(q / plane);
  const long long r = q - (long long)k * plane;
  const int j = (int)(r / P.gnx), i = (int)(r - (long long)j * P.gnx);
  px = P.gx + (T(i) + T(0.5)) * P.h;
  py = P.gy + (T(j) + T(0.5)) * P.h;
  pz = P.gz + (T(k) + T(0.5)) * P.h;
}

template <typename T>
__device__ __forceinline__ Tri<T> load_tri(const SdfParams<T> &P, int t) {
  // the caller checks the faces (the Python layer does, before the upload); an index out of
  // range is clamped to vertex 0 here so that no access leaves the vertex array
  int id[3];
  for (int c = 0; c < 3; ++c) {
    const int v = P.faces[3 * t + c];
    id[c] = (v < 0 || v >= P.nvert) ? 0 : v;
  }
  const T *a = P.verts + 3 * (size_t)id[0], *b = P.verts + 3 * (size_t)id[1], *c = P.verts + 3 * (size_t)id[2];
  Tri<T> r{a[0], a[1], a[2], b[0], b[1], b[2], c[0], c[1], c[2], T(0), T(0), T(0), T(0)};
  r.mx = (r.ax + r.bx + r.cx) * T(1.0 / 3.0);
  r.my = (r.ay + r.by + r.cy) * T(1.0 / 3.0);
  r.mz = (r.az + r.bz + r.cz) * T(1.0 / 3.0);
  auto d2 = [&](T x, T y, T z) { return (x - r.mx) * (x - r.mx) + (y - r.my) * (y - r.my) + (z - r.mz) * (z - r.mz); };
  T r2 = d2(r.ax, r.ay, r.az);
  r2 = fmax(r2, d2(r.bx, r.by, r.bz));
  r2 = fmax(r2, d2(r.cx, r.cy, r.cz));
  r.rad = sqrt(r2);
  return r;
}

// nearest triangle, winding number, distance, plane distance and the face votes
template <typename T>
__global__ void __launch_bounds__(NT) sdf_search_kernel(const __grid_constant__ SdfParams<T> P) {
  aero::pdl_wait();
  __shared__ Tri<T> S[TCH];
  const long long q = (long long)blockIdx.x * NT + threadIdx.x;
  const bool live = q < P.npt;
  T px = T(0), py = T(0), pz = T(0);
  if (live) point_of<T>(P, q, px, py, pz);
  T dmin = std::numeric_limits<T>::infinity();  // nearest so far: the first index of the minimum
  T smin = dmin;                                // its square root, for the ball test
  int imin = 0;
  T wsum = T(0);
  for (int t0 = 0; t0 < P.nface; t0 += TCH) {
    const int n = P.nface - t0 < TCH ? P.nface - t0 : TCH;
    __syncthreads();
    for (int e = threadIdx.x; e < n; e += NT) S[e] = load_tri<T>(P, t0 + e);
    __syncthreads();
    if (live) {
      T ws = T(0);
      for (int e = 0; e < n; ++e) {
        const Tri<T> t = S[e];
        // the triangle lies in its ball, so its distance is at least |p - m| - rad; when that
        // exceeds the nearest distance so far (with a 5e-5 relative margin for rounding) it
        // cannot be the nearest and its exact distance is skipped.  The winding number still
        // takes every triangle.
        const T qx = px - t.mx, qy = py - t.my, qz = pz - t.mz;
        const T lim = smin + t.rad;
        if (!(qx * qx + qy * qy + qz * qz > lim * lim * T(1.0001))) {
          const T d2 = tri_d2<T>(px, py, pz, t);
          if (d2 < dmin) {
            dmin = d2;
            smin = sqrt(d2);
            imin = t0 + e;
          }
        }
        ws += solid_angle<T>(px, py, pz, t);
      }
      wsum += ws;
    }
  }
  if (!live) return;
  const bool inside = fabs(wsum) > T(2.0 * 3.14159265358979323846);
  const Tri<T> t = load_tri<T>(P, imin);
  const T d2 = dmin;
  const T lim = T(1e-24);
  const T d = sqrt(d2 > lim ? d2 : lim);
  const T e0x = t.bx - t.ax, e0y = t.by - t.ay, e0z = t.bz - t.az;
  const T e1x = t.cx - t.ax, e1y = t.cy - t.ay, e1z = t.cz - t.az;
  const T nx = e0y * e1z - e0z * e1y, ny = e0z * e1x - e0x * e1z, nz = e0x * e1y - e0y * e1x;
  T nn = (nx * nx + ny * ny) + nz * nz;
  const T tiny = std::numeric_limits<T>::min();
  nn = nn > tiny ? nn : tiny;
  const T dp = ((nx * (px - t.ax) + ny * (py - t.ay)) + nz * (pz - t.az)) / sqrt(nn);
  const bool in_plane = (d2 - dp * dp) <= T(1e-18) + T(1e-12) * d2;
  if (in_plane && fabs(dp) > P.zone && dp != T(0)) atomicAdd(P.votes + imin, (inside ? -1 : 1) * (dp > T(0) ? 1 : -1));
  P.best[q] = imin;
  P.flag[q] = (unsigned char)((inside ? 1 : 0) | (in_plane ? 2 : 0));
  P.dist[q] = d;
  P.dpl[q] = dp;
}

// the mesh's orientation: sign of sum a . (b x c) over its triangles (FP64, one block)
template <typename T>
__global__ void orient_kernel(const __grid_constant__ SdfParams<T> P, int *orient) {
  aero::pdl_wait();
  __shared__ double red[NT / 32];
  double s = 0.0;
  for (int t = threadIdx.x; t < P.nface; t += NT) {
    const Tri<T> q = load_tri<T>(P, t);
    const double ax = q.ax, ay = q.ay, az = q.az, bx = q.bx, by = q.by, bz = q.bz, cx = q.cx, cy = q.cy, cz = q.cz;
    s += ax * (by * cz - bz * cy) + ay * (bz * cx - bx * cz) + az * (bx * cy - by * cx);
  }
  s = warp_sum(s);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double tot = 0.0;
    for (int w = 0; w < NT / 32; ++w) tot += red[w];
    *orient = tot > 0.0 ? 1 : (tot < 0.0 ? -1 : 0);
  }
}

template <typename T>
__global__ void __launch_bounds__(NT) sdf_finish_kernel(const __grid_constant__ SdfParams<T> P) {
  aero::pdl_wait();
  const long long q = (long long)blockIdx.x * NT + threadIdx.x;
  if (q >= P.npt) return;
  if (P.nface == 0) {  // no surface: everything is outside, at no finite distance
    P.out[q] = std::numeric_limits<T>::infinity();
    return;
  }
  const int b = P.best[q];
  const unsigned char fl = P.flag[q];
  const T sig = (fl & 1) ? T(-1) : T(1);
  const T dp = P.dpl[q];
  const int v = P.votes[b];
  const int side = v != 0 ? (v > 0 ? 1 : -1) : *P.orient;
  const bool on = (fl & 2) && fabs(dp) <= P.zone && side != 0;
  P.out[q] = on ? T(side) * dp : sig * P.dist[q];
}

// ---- assembly of one staggered grid (geometry.py:409-494)
template <typename T>
struct AssembleParams {
  int g;                      // 0 u, 1 v, 2 w, 3 cells
  int nx, ny, nz;             // points of this grid: x fastest
  T ox, oy, oz, h;            // origin of the first centre minus h / 2
  T w, shift;                 // ramp half-width, wall shift
  int zero_lo, zero_hi;       // boundary faces along the grid's normal axis to zero
  int nb;
  const T *sdf;               // (nb, npt)
  T om[AERO_MAX_BODIES], cx[AERO_MAX_BODIES], cy[AERO_MAX_BODIES], cz[AERO_MAX_BODIES];
  T axx[AERO_MAX_BODIES], axy[AERO_MAX_BODIES], axz[AERO_MAX_BODIES];
  T xr, yr, zr;
  T *chi, *a, *k;             // (npt), (npt), (nb, 3, npt); a and k NULL for the cells
};

template <typename T>
__global__ void __launch_bounds__(NT) assemble_kernel(const __grid_constant__ AssembleParams<T> P) {
  aero::pdl_wait();
  const long long npt = (long long)P.nx * P.ny * P.nz;
  const long long q = (long long)blockIdx.x * NT + threadIdx.x;
  if (q >= npt) return;
  const long long plane = (long long)P.nx * P.ny;
  const int k = (int)(q / plane);
  const long long r = q - (long long)k * plane;
  const int j = (int)(r / P.nx), i = (int)(r - (long long)j * P.nx);
  const T x = P.ox + (T(i) + T(0.5)) * P.h, y = P.oy + (T(j) + T(0.5)) * P.h, z = P.oz + (T(k) + T(0.5)) * P.h;
  const int along = P.g == 0 ? i : (P.g == 1 ? j : k);
  const int last = P.g == 0 ? P.nx - 1 : (P.g == 1 ? P.ny - 1 : P.nz - 1);
  const bool zero = P.g < 3 && ((P.zero_lo && along == 0) || (P.zero_hi && along == last));
  T c[AERO_MAX_BODIES];
  T sum = T(0), av = T(0);
  const T half_pi = T(0.5 * 3.14159265358979323846);
  for (int b = 0; b < P.nb; ++b) {
    T s = (P.sdf[(size_t)b * npt + q] + P.shift) / P.w;
    s = s > T(-1) ? (s < T(1) ? s : T(1)) : T(-1);
    T cb = T(0.5) - T(0.5) * sin(half_pi * s);
    if (zero) cb = cb * T(0);
    c[b] = cb;
    sum = b == 0 ? cb : sum + cb;
    if (P.g < 3 && P.om[b] != T(0)) {
      T rot;
      if (P.g == 0) rot = P.axy[b] * (z - P.cz[b]) - P.axz[b] * (y - P.cy[b]);
      else if (P.g == 1) rot = P.axz[b] * (x - P.cx[b]) - P.axx[b] * (z - P.cz[b]);
      else rot = P.axx[b] * (y - P.cy[b]) - P.axy[b] * (x - P.cx[b]);
      av = av + cb * (P.om[b] * rot);
    }
  }
  P.chi[q] = sum < T(1) ? sum : T(1);
  if (P.g == 3) return;
  P.a[q] = av;
  const T den = sum + T(1e-30);
  for (int b = 0; b < P.nb; ++b) {
    const T wb = P.nb == 1 ? T(1) : c[b] / den;
    T k1, k2;
    if (P.g == 0) {
      k1 = wb * (z - P.zr);
      k2 = -wb * (y - P.yr);
    } else if (P.g == 1) {
      k1 = -wb * (z - P.zr);
      k2 = wb * (x - P.xr);
    } else {
      k1 = wb * (y - P.yr);
      k2 = -wb * (x - P.xr);
    }
    T *kb = P.k + (size_t)b * 3 * npt;
    kb[q] = wb;
    kb[npt + q] = k1;
    kb[2 * npt + q] = k2;
  }
}

}  // namespace masks
}  // namespace aero

namespace {

using aero_host::align_up;
using aero_host::set_error;

// workspace of one signed-distance pass: best, flag, dist, dpl (npt), votes (nface), orient, bad
size_t sdf_scratch_bytes(size_t esz, long long npt, int nface) {
  return align_up(sizeof(int) * npt) + align_up(npt) + 2 * align_up(esz * npt) + align_up(sizeof(int) * (nface + 1)) +
         align_up(2 * sizeof(int));
}

template <typename T>
int sdf_pass(const T *verts, int nvert, const int32_t *faces, int nface, const T *pts, long long npt, int gnx, int gny,
             const double org[3], double h, double zone, T *out, unsigned char *ws, cudaStream_t s) {
  using namespace aero::masks;
  if (npt == 0) return AERO_OK;
  SdfParams<T> P{};
  P.verts = verts;
  P.nvert = nvert;
  P.faces = faces;
  P.nface = nface;
  P.pts = pts;
  P.npt = npt;
  P.gnx = gnx;
  P.gny = gny;
  if (!pts) {
    P.gx = T(org[0]);
    P.gy = T(org[1]);
    P.gz = T(org[2]);
    P.h = T(h);
  }
  P.zone = T(zone);
  size_t off = 0;
  auto take = [&](size_t bytes) {
    unsigned char *p = ws + off;
    off += align_up(bytes);
    return p;
  };
  P.best = reinterpret_cast<int *>(take(sizeof(int) * npt));
  P.flag = take(npt);
  P.dist = reinterpret_cast<T *>(take(sizeof(T) * npt));
  P.dpl = reinterpret_cast<T *>(take(sizeof(T) * npt));
  P.votes = reinterpret_cast<int *>(take(sizeof(int) * (nface + 1)));
  int *misc = reinterpret_cast<int *>(take(2 * sizeof(int)));
  P.orient = misc;
  P.out = out;
  const unsigned blocks = (unsigned)((npt + NT - 1) / NT);
  if (nface > 0) {
    AERO_CUDA_TRY(cudaMemsetAsync(P.votes, 0, sizeof(int) * (nface + 1), s));
    AERO_CUDA_TRY(cudaMemsetAsync(misc, 0, 2 * sizeof(int), s));
    (void)aero::launch_k(orient_kernel<T>, 1, NT, 0, s, P, misc);
    AERO_CUDA_TRY(cudaGetLastError());
    (void)aero::launch_k(sdf_search_kernel<T>, blocks, NT, 0, s, P);
    AERO_CUDA_TRY(cudaGetLastError());
  }
  (void)aero::launch_k(sdf_finish_kernel<T>, blocks, NT, 0, s, P);
  AERO_CUDA_TRY(cudaGetLastError());
  return AERO_OK;
}

bool window_ok(const AeroMaskConfig &c) {
  const int *w = c.window;
  return w[0] >= 0 && w[1] <= c.nz && w[2] >= 0 && w[3] <= c.ny && w[4] >= 0 && w[5] <= c.nx && w[1] > w[0] &&
         w[3] > w[2] && w[5] > w[4];
}

// points of grid g (u, v, w, cells) over the window: (nx, ny, nz)
void grid_dims(const AeroMaskConfig &c, int g, long long d[3]) {
  const long long wz = c.window[1] - c.window[0], wy = c.window[3] - c.window[2], wx = c.window[5] - c.window[4];
  d[0] = wx + (g == 0);
  d[1] = wy + (g == 1);
  d[2] = wz + (g == 2);
}

int check_config(const AeroMaskConfig *cfg, const AeroMaskBody *bodies) {
  if (!cfg) return set_error(AERO_EINVAL, "null argument");
  const AeroMaskConfig &c = *cfg;
  if (c.abi_version != AERO_ABI_VERSION) return set_error(AERO_EINVAL, "ABI version mismatch");
  if (c.dtype != AERO_F32 && c.dtype != AERO_F64) return set_error(AERO_EINVAL, "dtype must be float32 or float64");
  if (c.nbody < 1 || c.nbody > AERO_MAX_BODIES)
    return set_error(AERO_EUNSUPPORTED, "1 to " + std::to_string(AERO_MAX_BODIES) + " bodies");
  if (!bodies) return set_error(AERO_EINVAL, "null bodies");
  if (!(c.h > 0) || !(c.mask_width > 0)) return set_error(AERO_EINVAL, "h and mask_width must be positive");
  if (!window_ok(c)) return set_error(AERO_EINVAL, "empty window or window outside the domain");
  for (int b = 0; b < c.nbody; ++b)
    if (bodies[b].nface < 0 || bodies[b].nvert < 0 || (bodies[b].nface > 0 && (!bodies[b].vertices || !bodies[b].faces)))
      return set_error(AERO_EINVAL, "body mesh pointers or sizes invalid");
  return AERO_OK;
}

template <typename T>
int build_impl(const AeroMaskConfig &c, const AeroMaskBody *bodies, const AeroMaskOut *o, unsigned char *ws,
               cudaStream_t s) {
  using namespace aero::masks;
  const double h = c.h;
  const double X0 = c.x0 + c.window[4] * h, Y0 = c.y0 + c.window[2] * h, Z0 = c.z0 + c.window[0] * h;
  // origins of the four grids (geometry.py:409-415): faces half a cell before the window
  const double org[4][3] = {{X0 - 0.5 * h, Y0, Z0}, {X0, Y0 - 0.5 * h, Z0}, {X0, Y0, Z0 - 0.5 * h}, {X0, Y0, Z0}};
  long long maxpt = 0;
  for (int g = 0; g < 4; ++g) {
    long long d[3];
    grid_dims(c, g, d);
    maxpt = std::max(maxpt, d[0] * d[1] * d[2]);
  }
  T *sdf = reinterpret_cast<T *>(ws);
  unsigned char *scratch = ws + align_up(sizeof(T) * (size_t)c.nbody * maxpt);
  void *chi[4] = {o->chi_u, o->chi_v, o->chi_w, o->chi_c};
  void *av[3] = {o->a_u, o->a_v, o->a_w};
  void *kv[3] = {o->k_u, o->k_v, o->k_w};
  const int lo[3] = {c.window[4] == 0, c.window[2] == 0, c.window[0] == 0};
  const int hi[3] = {c.window[5] == c.nx, c.window[3] == c.ny, c.window[1] == c.nz};
  for (int g = 0; g < 4; ++g) {
    long long d[3];
    grid_dims(c, g, d);
    const long long npt = d[0] * d[1] * d[2];
    for (int b = 0; b < c.nbody; ++b) {
      const int rc = sdf_pass<T>(static_cast<const T *>(bodies[b].vertices), bodies[b].nvert, bodies[b].faces,
                                 bodies[b].nface, nullptr, npt, (int)d[0], (int)d[1], org[g], h, 0.02 * h,
                                 sdf + (size_t)b * npt, scratch, s);
      if (rc) return rc;
    }
    AssembleParams<T> A{};
    A.g = g;
    A.nx = (int)d[0];
    A.ny = (int)d[1];
    A.nz = (int)d[2];
    A.ox = T(org[g][0]);
    A.oy = T(org[g][1]);
    A.oz = T(org[g][2]);
    A.h = T(h);
    A.w = T(c.mask_width * h);
    A.shift = T(c.mask_shift * h);
    if (g < 3 && !c.periodic[g]) {
      A.zero_lo = lo[g];
      A.zero_hi = hi[g];
    }
    A.nb = c.nbody;
    A.sdf = sdf;
    for (int b = 0; b < c.nbody; ++b) {
      A.om[b] = T(bodies[b].omega);
      A.cx[b] = T(bodies[b].center[0]);
      A.cy[b] = T(bodies[b].center[1]);
      A.cz[b] = T(bodies[b].center[2]);
      A.axx[b] = T(bodies[b].axis[0]);
      A.axy[b] = T(bodies[b].axis[1]);
      A.axz[b] = T(bodies[b].axis[2]);
    }
    A.xr = T(c.moment_ref[0]);
    A.yr = T(c.moment_ref[1]);
    A.zr = T(c.moment_ref[2]);
    A.chi = static_cast<T *>(chi[g]);
    A.a = g < 3 ? static_cast<T *>(av[g]) : nullptr;
    A.k = g < 3 ? static_cast<T *>(kv[g]) : nullptr;
    (void)aero::launch_k(assemble_kernel<T>, (unsigned)((npt + NT - 1) / NT), NT, 0, s, A);
    AERO_CUDA_TRY(cudaGetLastError());
  }
  return AERO_OK;
}

}  // namespace

extern "C" {

size_t aero_ns3d_masks_workspace_bytes(const AeroMaskConfig *cfg, const AeroMaskBody *bodies) {
  if (check_config(cfg, bodies)) return 0;
  const AeroMaskConfig &c = *cfg;
  const size_t e = c.dtype == AERO_F64 ? 8 : 4;
  long long maxpt = 0;
  int maxface = 0;
  for (int g = 0; g < 4; ++g) {
    long long d[3];
    grid_dims(c, g, d);
    maxpt = std::max(maxpt, d[0] * d[1] * d[2]);
  }
  for (int b = 0; b < c.nbody; ++b) maxface = std::max(maxface, bodies[b].nface);
  return align_up(e * (size_t)c.nbody * maxpt) + sdf_scratch_bytes(e, maxpt, maxface);
}

int aero_ns3d_build_masks(const AeroMaskConfig *cfg, const AeroMaskBody *bodies, const AeroMaskOut *out,
                          void *workspace, void *stream) {
  const int rc = check_config(cfg, bodies);
  if (rc) return rc;
  if (!out || !workspace) return set_error(AERO_EINVAL, "null argument");
  if (!out->chi_u || !out->chi_v || !out->chi_w || !out->chi_c || !out->a_u || !out->a_v || !out->a_w || !out->k_u ||
      !out->k_v || !out->k_w)
    return set_error(AERO_EINVAL, "missing mask output");
  if (reinterpret_cast<uintptr_t>(workspace) % aero_host::ALIGN)
    return set_error(AERO_EINVAL, "workspace must be 256-byte aligned");
  auto s = static_cast<cudaStream_t>(stream);
  auto ws = static_cast<unsigned char *>(workspace);
  return cfg->dtype == AERO_F64 ? build_impl<double>(*cfg, bodies, out, ws, s) : build_impl<float>(*cfg, bodies, out, ws, s);
}

size_t aero_mesh_sdf_workspace_bytes(int32_t dtype, int32_t nface, int64_t npoints) {
  if ((dtype != AERO_F32 && dtype != AERO_F64) || nface < 0 || npoints < 0) return 0;
  return sdf_scratch_bytes(dtype == AERO_F64 ? 8 : 4, npoints, nface);
}

int aero_mesh_signed_distance(int32_t dtype, const void *vertices, int32_t nvert, const int32_t *faces, int32_t nface,
                              const void *points, int64_t npoints, double plane_zone, void *out, void *workspace,
                              void *stream) {
  if (dtype != AERO_F32 && dtype != AERO_F64) return set_error(AERO_EINVAL, "dtype must be float32 or float64");
  if (nface < 0 || nvert < 0 || npoints < 0) return set_error(AERO_EINVAL, "negative size");
  if (npoints > 0 && (!points || !out || !workspace)) return set_error(AERO_EINVAL, "null argument");
  if (nface > 0 && (!vertices || !faces)) return set_error(AERO_EINVAL, "null mesh");
  if (reinterpret_cast<uintptr_t>(workspace) % aero_host::ALIGN)
    return set_error(AERO_EINVAL, "workspace must be 256-byte aligned");
  auto s = static_cast<cudaStream_t>(stream);
  auto ws = static_cast<unsigned char *>(workspace);
  const double org[3] = {0.0, 0.0, 0.0};
  if (dtype == AERO_F64)
    return sdf_pass<double>(static_cast<const double *>(vertices), nvert, faces, nface,
                            static_cast<const double *>(points), npoints, 0, 0, org, 0.0, plane_zone,
                            static_cast<double *>(out), ws, s);
  return sdf_pass<float>(static_cast<const float *>(vertices), nvert, faces, nface, static_cast<const float *>(points),
                         npoints, 0, 0, org, 0.0, plane_zone, static_cast<float *>(out), ws, s);
}

}  // extern "C"
