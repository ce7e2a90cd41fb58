// Epilogue helpers shared by the angular kernels of both forms: density multipoles and
// dipole/acceleration partial sums of one orbital column over one tile of radii.  The shared-memory
// orbitals may be complex128 (FP64 form) or complex64 (split form); products and sums are FP64.
#pragma once
#include "ggb_internal.cuh"

namespace ggb {

__device__ __forceinline__ double2 to_d2(double2 v) { return v; }
__device__ __forceinline__ double2 to_d2(float2 v) { return make_double2((double)v.x, (double)v.y); }

__device__ __forceinline__ double cf(const double* tab, int n_l, int l) {
  return (l >= 0 && l < n_l) ? tab[l] : 0.0;
}

template <class C, int STRIDE = TR>
__device__ __forceinline__ double xdot(const C* xs, int n_l, int a, int b, int lane) {
  if (a < 0 || a >= n_l || b < 0 || b >= n_l) return 0.0;
  const C xa = xs[a * STRIDE + lane];
  const C xb = xs[b * STRIDE + lane];
  return (double)xa.x * (double)xb.x + (double)xa.y * (double)xb.y;
}

// One multipole of one orbital's density at one radius, with the reference's literal l ranges
// (hartreePotentialDensity.cuh:21-177, including the tail loop of L = 3 that restarts at N_l-4).
template <class C, int STRIDE = TR>
__device__ double density_multipole(int L, int m, int n_l, const C* xs, int lane,
                                    const double* coef, int n_m) {
  const double* cu = coef + ((size_t)CF_CU * n_m + m) * n_l;
  const double* cd = coef + ((size_t)CF_CD * n_m + m) * n_l;
  const double* pp = coef + ((size_t)CF_P * n_m + m) * n_l;
  const double* qu = coef + ((size_t)CF_QU * n_m + m) * n_l;
  const double* qd = coef + ((size_t)CF_QD * n_m + m) * n_l;
  const double* p3 = coef + ((size_t)CF_P3 * n_m + m) * n_l;
  const double* f3 = coef + ((size_t)CF_F3 * n_m + m) * n_l;
  double d = 0.0;
  if (L == 0) {
    for (int lp = m; lp < n_l; ++lp) {
      const C v = xs[lp * STRIDE + lane];
      d += (double)v.x * (double)v.x + (double)v.y * (double)v.y;
    }
  } else if (L == 1) {
    int lp = m;
    d += cf(cu, n_l, lp) * xdot<C, STRIDE>(xs, n_l, lp + 1, lp, lane);
    for (lp = m + 1; lp < n_l - 1; ++lp)
      d += cf(cu, n_l, lp) * xdot<C, STRIDE>(xs, n_l, lp + 1, lp, lane) + cf(cd, n_l, lp) * xdot<C, STRIDE>(xs, n_l, lp - 1, lp, lane);
    lp = n_l - 1;
    d += cf(cd, n_l, lp) * xdot<C, STRIDE>(xs, n_l, lp - 1, lp, lane);
  } else if (L == 2) {
    for (int lp = m; lp < m + 2; ++lp)
      d += cf(qu, n_l, lp) * xdot<C, STRIDE>(xs, n_l, lp + 2, lp, lane) + cf(pp, n_l, lp) * xdot<C, STRIDE>(xs, n_l, lp, lp, lane);
    for (int lp = m + 2; lp < n_l - 2; ++lp)
      d += cf(qu, n_l, lp) * xdot<C, STRIDE>(xs, n_l, lp + 2, lp, lane) + cf(qd, n_l, lp) * xdot<C, STRIDE>(xs, n_l, lp - 2, lp, lane) +
           cf(pp, n_l, lp) * xdot<C, STRIDE>(xs, n_l, lp, lp, lane);
    for (int lp = n_l - 2; lp < n_l; ++lp)
      d += cf(qd, n_l, lp) * xdot<C, STRIDE>(xs, n_l, lp - 2, lp, lane) + cf(pp, n_l, lp) * xdot<C, STRIDE>(xs, n_l, lp, lp, lane);
  } else if (L == 3) {
    int lp = m;
    d += cf(p3, n_l, lp) * xdot<C, STRIDE>(xs, n_l, lp + 1, lp, lane) + cf(f3, n_l, lp) * xdot<C, STRIDE>(xs, n_l, lp + 3, lp, lane);
    for (lp = m + 1; lp < m + 3; ++lp)
      d += cf(p3, n_l, lp - 1) * xdot<C, STRIDE>(xs, n_l, lp - 1, lp, lane) + cf(p3, n_l, lp) * xdot<C, STRIDE>(xs, n_l, lp + 1, lp, lane) +
           cf(f3, n_l, lp) * xdot<C, STRIDE>(xs, n_l, lp + 3, lp, lane);
    for (lp = m + 3; lp < n_l - 3; ++lp)
      d += cf(f3, n_l, lp - 3) * xdot<C, STRIDE>(xs, n_l, lp - 3, lp, lane) + cf(p3, n_l, lp - 1) * xdot<C, STRIDE>(xs, n_l, lp - 1, lp, lane) +
           cf(p3, n_l, lp) * xdot<C, STRIDE>(xs, n_l, lp + 1, lp, lane) + cf(f3, n_l, lp) * xdot<C, STRIDE>(xs, n_l, lp + 3, lp, lane);
    for (lp = n_l - 4; lp < n_l - 1; ++lp)
      d += cf(f3, n_l, lp - 3) * xdot<C, STRIDE>(xs, n_l, lp - 3, lp, lane) + cf(p3, n_l, lp - 1) * xdot<C, STRIDE>(xs, n_l, lp - 1, lp, lane) +
           cf(p3, n_l, lp) * xdot<C, STRIDE>(xs, n_l, lp + 1, lp, lane);
    d += cf(f3, n_l, lp - 3) * xdot<C, STRIDE>(xs, n_l, lp - 3, lp, lane) + cf(p3, n_l, lp - 1) * xdot<C, STRIDE>(xs, n_l, lp - 1, lp, lane);
  }
  return d;
}

// compensated sum over aligned segments of `seg` lanes (seg = 32: the whole warp)
// The seven coefficient rows of one m (CF_CU .. CF_F3 order), contiguous: rows[c * n_l + l].
// Density multipoles L = 0 .. n_den-1 of one orbital at the radius of this lane: the same terms and
// literal l ranges as density_multipole, but every l loop is strided over the n_warps warps, and
// this warp's partial sums are added to d[L] (the caller sums the warps).  Coefficient c of this m
// is rows[c * row_stride + l] (row_stride 0: n_l, the rows contiguous).
template <class C, int STRIDE>
__device__ void density_partials(int n_den, int m, int n_l, const C* xs, int lane, const double* rows,
                                 int warp, int n_warps, double (&d)[N_DEN], int row_stride = 0) {
  const size_t rs = row_stride > 0 ? (size_t)row_stride : (size_t)n_l;
  const double* cu = rows + CF_CU * rs;
  const double* cd = rows + CF_CD * rs;
  const double* pp = rows + CF_P * rs;
  const double* qu = rows + CF_QU * rs;
  const double* qd = rows + CF_QD * rs;
  const double* p3 = rows + CF_P3 * rs;
  const double* f3 = rows + CF_F3 * rs;
  auto X = [&](int a, int b) { return xdot<C, STRIDE>(xs, n_l, a, b, lane); };
  // L = 0
  for (int lp = m + warp; lp < n_l; lp += n_warps) d[0] += X(lp, lp);
  if (n_den > 1) {
    if (warp == 0) d[1] += cf(cu, n_l, m) * X(m + 1, m);
    for (int lp = m + 1 + warp; lp < n_l - 1; lp += n_warps)
      d[1] += cf(cu, n_l, lp) * X(lp + 1, lp) + cf(cd, n_l, lp) * X(lp - 1, lp);
    if (warp == n_warps - 1) d[1] += cf(cd, n_l, n_l - 1) * X(n_l - 2, n_l - 1);
  }
  if (n_den > 2) {
    for (int lp = m + warp; lp < m + 2; lp += n_warps)
      d[2] += cf(qu, n_l, lp) * X(lp + 2, lp) + cf(pp, n_l, lp) * X(lp, lp);
    for (int lp = m + 2 + warp; lp < n_l - 2; lp += n_warps)
      d[2] += cf(qu, n_l, lp) * X(lp + 2, lp) + cf(qd, n_l, lp) * X(lp - 2, lp) + cf(pp, n_l, lp) * X(lp, lp);
    for (int lp = n_l - 2 + warp; lp < n_l; lp += n_warps)
      d[2] += cf(qd, n_l, lp) * X(lp - 2, lp) + cf(pp, n_l, lp) * X(lp, lp);
  }
  if (n_den > 3) {
    if (warp == 0) d[3] += cf(p3, n_l, m) * X(m + 1, m) + cf(f3, n_l, m) * X(m + 3, m);
    for (int lp = m + 1 + warp; lp < m + 3; lp += n_warps)
      d[3] += cf(p3, n_l, lp - 1) * X(lp - 1, lp) + cf(p3, n_l, lp) * X(lp + 1, lp) + cf(f3, n_l, lp) * X(lp + 3, lp);
    for (int lp = m + 3 + warp; lp < n_l - 3; lp += n_warps)
      d[3] += cf(f3, n_l, lp - 3) * X(lp - 3, lp) + cf(p3, n_l, lp - 1) * X(lp - 1, lp) + cf(p3, n_l, lp) * X(lp + 1, lp) +
              cf(f3, n_l, lp) * X(lp + 3, lp);
    // the reference's tail loop restarts at N_l - 4 (hartreePotentialDensity.cuh:150)
    for (int lp = n_l - 4 + warp; lp < n_l - 1; lp += n_warps)
      d[3] += cf(f3, n_l, lp - 3) * X(lp - 3, lp) + cf(p3, n_l, lp - 1) * X(lp - 1, lp) + cf(p3, n_l, lp) * X(lp + 1, lp);
    if (warp == n_warps - 1) {
      const int lp = n_l - 1;
      d[3] += cf(f3, n_l, lp - 3) * X(lp - 3, lp) + cf(p3, n_l, lp - 1) * X(lp - 1, lp);
    }
  }
}

__device__ __forceinline__ dd warp_sum_dd(double v, int seg = 32) {
  dd a{v, 0.0};
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    if (o < seg) {
      const dd b{__shfl_xor_sync(0xffffffffu, a.hi, o), __shfl_xor_sync(0xffffffffu, a.lo, o)};
      a = dd_add(a, b);
    }
  }
  return a;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Dipole and acceleration partial sums for every l of one column over the radii r0 + lane held by
// a lane group -- a warp, or half of one with seg = 16, the halves on different l
// (dipoleMoment.cuh:19-43 / dipoleAcceleration.cuh:17-41 followed by cublasZdotc): one
// partial per g.obs_seg consecutive radii (32 or 16), index (r0 + lane) / g.obs_seg.  Lanes from
// n_valid on hold no radius.
// COMPENSATED: double-double sums (the FP64 form, held to 1e-10 of the reference); otherwise plain
// FP64 sums (the split forms, whose own error is far larger than FP64 summation error).
// cu_row, cd_row: the c_u and c_d rows of this m when the caller has staged them (e.g. in shared
// memory); by default they are read from the group's table.
template <class C, int STRIDE = TR, bool COMPENSATED = true>
__device__ void observables_tile(const GroupArgs& g, const C* xs, int col, int m, int r0, int lane,
                                 int warp, int n_warps, double rr, double fr2, int n_valid = TR,
                                 const double* cu_row = nullptr, const double* cd_row = nullptr) {
  const int n_l = g.n_l;
  const int seg = g.obs_seg;
  const bool lv = lane < n_valid;
  const double* cu = cu_row ? cu_row : g.coef + ((size_t)CF_CU * g.n_m + m) * n_l;
  const double* cd = cd_row ? cd_row : g.coef + ((size_t)CF_CD * g.n_m + m) * n_l;
  // every lane runs the same number of iterations (the shuffles below span the whole warp, whose
  // lane groups may hold different l)
  const int iters = (n_l + n_warps - 1) / n_warps;
  for (int it = 0; it < iters; ++it) {
    const int l = warp + it * n_warps;
    const bool lok = l < n_l;
    double4 out = make_double4(0.0, 0.0, 0.0, 0.0);
    if (lok && l >= m && lv) {
      const double2 xl = to_d2(xs[l * STRIDE + lane]);
      const double2 xu = (l + 1 < n_l) ? to_d2(xs[(l + 1) * STRIDE + lane]) : make_double2(0.0, 0.0);
      const double2 xd = (l >= 1) ? to_d2(xs[(l - 1) * STRIDE + lane]) : make_double2(0.0, 0.0);
      const double c_u = cu[l], c_d = cd[l];
      double2 z1, z2;
      if (l == m) {
        z1 = make_double2(rr * c_u * xu.x, rr * c_u * xu.y);
        z2 = make_double2(fr2 * c_u * xu.x, fr2 * c_u * xu.y);
      } else if (l == n_l - 1) {
        z1 = make_double2(rr * c_d * xd.x, rr * c_d * xd.y);
        z2 = make_double2(fr2 * c_d * xd.x, fr2 * c_d * xd.y);
      } else {
        z1 = make_double2(rr * c_u * xu.x + rr * c_d * xd.x, rr * c_u * xu.y + rr * c_d * xd.y);
        z2 = make_double2(fr2 * (c_u * xu.x + c_d * xd.x), fr2 * (c_u * xu.y + c_d * xd.y));
      }
      // conj(x_l) . z
      out.x = xl.x * z1.x + xl.y * z1.y;
      out.y = xl.x * z1.y - xl.y * z1.x;
      out.z = xl.x * z2.x + xl.y * z2.y;
      out.w = xl.x * z2.y - xl.y * z2.x;
    }
    // compensated (double-double) reduction over the tile's radii
    dd sx, sy, sz, sw;
    if (COMPENSATED) {
      sx = warp_sum_dd(out.x, seg); sy = warp_sum_dd(out.y, seg);
      sz = warp_sum_dd(out.z, seg); sw = warp_sum_dd(out.w, seg);
    } else {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        if (o < seg) {
          out.x += __shfl_xor_sync(0xffffffffu, out.x, o); out.y += __shfl_xor_sync(0xffffffffu, out.y, o);
          out.z += __shfl_xor_sync(0xffffffffu, out.z, o); out.w += __shfl_xor_sync(0xffffffffu, out.w, o);
        }
      }
      sx = dd{out.x, 0.0}; sy = dd{out.y, 0.0}; sz = dd{out.z, 0.0}; sw = dd{out.w, 0.0};
    }
    if (lok && lv && (lane & (seg - 1)) == 0) {
      double4* o = g.obs + 2 * (((size_t)col * n_l + l) * g.n_tiles + (r0 + lane) / seg);
      o[0] = make_double4(sx.hi, sy.hi, sz.hi, sw.hi);
      o[1] = make_double4(sx.lo, sy.lo, sz.lo, sw.lo);
    }
  }
}


}  // namespace ggb
