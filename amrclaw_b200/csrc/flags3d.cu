// Device kernels of the 3D level flag arrays (flglvl.f, domprep.f, domshrink.f,
// domup.f, spest.f, flag2refine.f, bufnst.f, projec.f, shiftset.f, colate.f).
// Every kernel is a grid-stride loop over int8 cells; the arrays of a 128^3 level
// are about 2 MB, so each pass is a few microseconds of HBM time.
#include "flags3d.cuh"
#include <algorithm>

namespace amrb {

namespace {

constexpr int NGF = 2;  // num_ghost of the patch storage

// std::max / Fortran max argument order (the CPU restatement's)
__device__ __forceinline__ double dmax(double a, double b) { return (a < b) ? b : a; }

int blocks_for(long long n, int block) {
  return (int)std::max<long long>(1, std::min<long long>((n + block - 1) / block, 148LL * 32));
}

#define GRID_STRIDE(t, n) for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < (n); t += (long long)gridDim.x * blockDim.x)

__global__ void boxes_kernel(int8_t* a, LvlDims d, const LvlBox* boxes, int nbox, int mode) {
  const int b = blockIdx.y;
  if (b >= nbox) return;
  const LvlBox B = boxes[b];
  const int ni = B.i1 - B.i0 + 1, nj = B.j1 - B.j0 + 1, nk = B.k1 - B.k0 + 1;
  if (ni <= 0 || nj <= 0 || nk <= 0) return;
  const long long n = (long long)ni * nj * nk;
  GRID_STRIDE(t, n) {
    const int i = B.i0 + (int)(t % ni), j = B.j0 + (int)((t / ni) % nj), k = B.k0 + (int)(t / ((long long)ni * nj));
    int8_t& v = a[d.at(i, j, k)];
    if (mode == 0) v = 1;
    else if (v == 0) v = 3;
  }
}

// extend_borders: ring cells of the six faces (edges and corners excluded) copy a 1 of the adjacent interior cell
__global__ void extend_kernel(int8_t* a, LvlDims d) {
  const long long fx = (long long)d.js * d.ks, fy = (long long)d.is * d.ks, fz = (long long)d.is * d.js;
  GRID_STRIDE(t0, 2 * (fx + fy + fz)) {
    long long t = t0;
    int i, j, k, si, sj, sk;
    if (t < 2 * fx) {
      const bool hi = t >= fx; if (hi) t -= fx;
      j = 1 + (int)(t % d.js); k = 1 + (int)(t / d.js);
      i = hi ? d.is + 1 : 0; si = hi ? d.is : 1; sj = j; sk = k;
    } else if ((t -= 2 * fx) < 2 * fy) {
      const bool hi = t >= fy; if (hi) t -= fy;
      i = 1 + (int)(t % d.is); k = 1 + (int)(t / d.is);
      j = hi ? d.js + 1 : 0; sj = hi ? d.js : 1; si = i; sk = k;
    } else {
      t -= 2 * fy;
      const bool hi = t >= fz; if (hi) t -= fz;
      i = 1 + (int)(t % d.is); j = 1 + (int)(t / d.is);
      k = hi ? d.ks + 1 : 0; sk = hi ? d.ks : 1; si = i; sj = j;
    }
    if (a[d.at(si, sj, sk)] == 1) a[d.at(i, j, k)] = 1;
  }
}

// fill_edges_corners, edges: a ring edge cell becomes 1 where both face neighbours are 1
__global__ void edges_kernel(int8_t* a, LvlDims d) {
  const int is = d.is, js = d.js, ks = d.ks;
  GRID_STRIDE(t0, 4LL * (ks + is + js)) {
    long long t = t0;
    auto F = [&](int i, int j, int k) { return (int)a[d.at(i, j, k)]; };
    if (t < 4LL * ks) {
      const int k = 1 + (int)(t / 4), e = (int)(t % 4);
      if (e == 0 && F(0, 1, k) + F(1, 0, k) == 2) a[d.at(0, 0, k)] = 1;
      if (e == 1 && F(0, js, k) + F(1, js + 1, k) == 2) a[d.at(0, js + 1, k)] = 1;
      if (e == 2 && F(is, 0, k) + F(is + 1, 1, k) == 2) a[d.at(is + 1, 0, k)] = 1;
      if (e == 3 && F(is, js + 1, k) + F(is + 1, js, k) == 2) a[d.at(is + 1, js + 1, k)] = 1;
    } else if ((t -= 4LL * ks) < 4LL * is) {
      const int i = 1 + (int)(t / 4), e = (int)(t % 4);
      if (e == 0 && F(i, 0, 1) + F(i, 1, 0) == 2) a[d.at(i, 0, 0)] = 1;
      if (e == 1 && F(i, js, 0) + F(i, js + 1, 1) == 2) a[d.at(i, js + 1, 0)] = 1;
      if (e == 2 && F(i, 0, ks) + F(i, 1, ks + 1) == 2) a[d.at(i, 0, ks + 1)] = 1;
      if (e == 3 && F(i, js + 1, ks) + F(i, js, ks + 1) == 2) a[d.at(i, js + 1, ks + 1)] = 1;
    } else {
      t -= 4LL * is;
      const int j = 1 + (int)(t / 4), e = (int)(t % 4);
      if (e == 0 && F(0, j, 1) + F(1, j, 0) == 2) a[d.at(0, j, 0)] = 1;
      if (e == 1 && F(is, j, 0) + F(is + 1, j, 1) == 2) a[d.at(is + 1, j, 0)] = 1;
      if (e == 2 && F(0, j, ks) + F(1, j, ks + 1) == 2) a[d.at(0, j, ks + 1)] = 1;
      if (e == 3 && F(is + 1, j, ks) + F(is, j, ks + 1) == 2) a[d.at(is + 1, j, ks + 1)] = 1;
    }
  }
}

// fill_edges_corners, corners: one thread, after the edges
__global__ void corners_kernel(int8_t* a, LvlDims d) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  const int is = d.is, js = d.js, ks = d.ks;
  auto F = [&](int i, int j, int k) { return (int)a[d.at(i, j, k)]; };
  if (F(0, 0, 1) + F(0, 1, 0) + F(1, 0, 0) == 3) a[d.at(0, 0, 0)] = 1;
  if (F(is + 1, 0, 1) + F(is + 1, 1, 0) + F(is, 0, 0) == 3) a[d.at(is + 1, 0, 0)] = 1;
  if (F(0, js + 1, 1) + F(0, js, 0) + F(1, js + 1, 0) == 3) a[d.at(0, js + 1, 0)] = 1;
  if (F(is + 1, js + 1, 1) + F(is + 1, js, 0) + F(is, js + 1, 0) == 3) a[d.at(is + 1, js + 1, 0)] = 1;
  if (F(0, 0, ks) + F(0, 1, ks + 1) + F(1, 0, ks + 1) == 3) a[d.at(0, 0, ks + 1)] = 1;
  if (F(is + 1, 0, ks) + F(is + 1, 1, ks + 1) + F(is, 0, ks + 1) == 3) a[d.at(is + 1, 0, ks + 1)] = 1;
  if (F(0, js + 1, ks) + F(0, js, ks + 1) + F(1, js + 1, ks + 1) == 3) a[d.at(0, js + 1, ks + 1)] = 1;
  if (F(is + 1, js + 1, ks) + F(is + 1, js, ks + 1) + F(is, js + 1, ks + 1) == 3) a[d.at(is + 1, js + 1, ks + 1)] = 1;
}

__device__ __forceinline__ bool is_ring(const LvlDims& d, int i, int j, int k) {
  return i == 0 || j == 0 || k == 0 || i == d.is + 1 || j == d.js + 1 || k == d.ks + 1;
}

// every cell of `out`: 0 on the ring, interior kept where all 27 cells of `in` are positive
__global__ void shrink_kernel(const int8_t* in, int8_t* out, LvlDims d) {
  GRID_STRIDE(t, d.size()) {
    const int i = (int)(t % (d.is + 2)), j = (int)((t / (d.is + 2)) % (d.js + 2)), k = (int)(t / ((long long)(d.is + 2) * (d.js + 2)));
    int8_t v = 0;
    if (!is_ring(d, i, j, k)) {
      bool ok = true;
      for (int c = -1; c <= 1 && ok; ++c)
        for (int b = -1; b <= 1 && ok; ++b) {
          const int8_t* row = in + d.at(i - 1, j + b, k + c);
          if (row[0] <= 0 || row[1] <= 0 || row[2] <= 0) ok = false;
        }
      v = ok ? in[t] : (int8_t)0;
    }
    out[t] = v;
  }
}

// every cell of `fine`: 0 on the ring, the covering coarse cell's value inside
__global__ void up_kernel(const int8_t* c, LvlDims cd, int8_t* f, LvlDims fd, int rx, int ry, int rz) {
  GRID_STRIDE(t, fd.size()) {
    const int i = (int)(t % (fd.is + 2)), j = (int)((t / (fd.is + 2)) % (fd.js + 2)), k = (int)(t / ((long long)(fd.is + 2) * (fd.js + 2)));
    f[t] = is_ring(fd, i, j, k) ? (int8_t)0 : c[cd.at((i - 1) / rx + 1, (j - 1) / ry + 1, (k - 1) / rz + 1)];
  }
}

__global__ void zero_interior_kernel(int8_t* f, LvlDims d) {
  GRID_STRIDE(t, (long long)d.is * d.js * d.ks) {
    const int i = 1 + (int)(t % d.is), j = 1 + (int)((t / d.is) % d.js), k = 1 + (int)(t / ((long long)d.is * d.js));
    f[d.at(i, j, k)] = 0;
  }
}

__global__ void zero_ring_kernel(int8_t* f, LvlDims d) {
  GRID_STRIDE(t, d.size()) {
    const int i = (int)(t % (d.is + 2)), j = (int)((t / (d.is + 2)) % (d.js + 2)), k = (int)(t / ((long long)(d.is + 2) * (d.js + 2)));
    if (is_ring(d, i, j, k)) f[t] = 0;
  }
}

// Binary search of the patch that holds level cell t.
__device__ __forceinline__ int patch_of(const long long* pre, int np, long long t) {
  int lo = 0, hi = np - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (pre[mid] <= t) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// flag2refine.f pattern of the 3D Euler example: undivided pressure difference (or of every
// component) against tolsp; BADPT (2) / GOODPT (0) into the zeroed level array (setflags.f)
template <class T>
__global__ void flag_cells_kernel(const T* pool, const PatchDev* patches, const int* plist, const long long* cell0, int np,
                                  long long ncells, int flag_pressure, double gamma1, double tolsp, int nvar, int8_t* f, LvlDims d) {
  GRID_STRIDE(t, ncells) {
    const int pi = patch_of(cell0, np, t);
    const PatchDev& P = patches[plist[pi]];
    const int mx = P.ihi - P.ilo + 1, my = P.jhi - P.jlo + 1;
    const long long loc = t - cell0[pi];
    const int i = (int)(loc % mx) + 1, j = (int)((loc / mx) % my) + 1, k = (int)(loc / ((long long)mx * my)) + 1;
    const long long plane = (long long)P.mitot * P.mjtot * P.mktot;
    const T* q = pool + P.q[P.cur];
    auto Q = [&](int m, int ii, int jj, int kk) {
      return q[(m - 1) * plane + ((long long)(kk - 1 + NGF) * P.mjtot + (jj - 1 + NGF)) * P.mitot + (ii - 1 + NGF)];
    };
    double dq = 0.0;
    if (flag_pressure) {
      auto pres = [&](int a, int b, int c) {
        const double rho = Q(1, a, b, c), mu = Q(2, a, b, c), mv = Q(3, a, b, c), mw = Q(4, a, b, c);
        return gamma1 * (Q(5, a, b, c) - 0.5 * (mu * mu + mv * mv + mw * mw) / rho);
      };
      const double dpi = fabs(pres(i + 1, j, k) - pres(i - 1, j, k));
      const double dpj = fabs(pres(i, j + 1, k) - pres(i, j - 1, k));
      const double dpk = fabs(pres(i, j, k + 1) - pres(i, j, k - 1));
      dq = dmax(dmax(dmax(dq, dpi), dpj), dpk);
    } else {
      for (int m = 1; m <= nvar; ++m) {
        const double dqi = fabs(Q(m, i + 1, j, k) - Q(m, i - 1, j, k));
        const double dqj = fabs(Q(m, i, j + 1, k) - Q(m, i, j - 1, k));
        const double dqk = fabs(Q(m, i, j, k + 1) - Q(m, i, j, k - 1));
        dq = dmax(dmax(dmax(dq, dqi), dqj), dqk);
      }
    }
    f[d.at(P.ilo + i, P.jlo + j, P.klo + k)] = (dq > tolsp) ? (int8_t)2 : (int8_t)0;
  }
}

// shiftset.f: every positive flag, in (k, j, i) order, stamps its value on the box of
// half-width b around it; the value a cell ends with is that of the lexicographically
// last (k, j, i) source within b in every direction. Three separable passes:
// t1(i, j, k) = last source along i (rows j, k interior, i over the whole array width)
__global__ void shift_i_kernel(const int8_t* f, int8_t* t1, LvlDims d, int b) {
  GRID_STRIDE(t, (long long)(d.is + 2) * d.js * d.ks) {
    const int i = (int)(t % (d.is + 2)), j = 1 + (int)((t / (d.is + 2)) % d.js), k = 1 + (int)(t / ((long long)(d.is + 2) * d.js));
    int8_t v = 0;
    for (int s = min(i + b, d.is); s >= max(i - b, 1); --s) {
      const int8_t x = f[d.at(s, j, k)];
      if (x > 0) { v = x; break; }
    }
    t1[d.at(i, j, k)] = v;
  }
}
// t2(i, j, k) = t1 of the last row j' within b that holds a source (k interior)
__global__ void shift_j_kernel(const int8_t* t1, int8_t* t2, LvlDims d, int b) {
  GRID_STRIDE(t, (long long)(d.is + 2) * (d.js + 2) * d.ks) {
    const int i = (int)(t % (d.is + 2)), jj = (int)((t / (d.is + 2)) % (d.js + 2)), k = 1 + (int)(t / ((long long)(d.is + 2) * (d.js + 2)));
    int8_t v = 0;
    for (int j = min(jj + b, d.js); j >= max(jj - b, 1); --j) {
      const int8_t x = t1[d.at(i, j, k)];
      if (x > 0) { v = x; break; }
    }
    t2[d.at(i, jj, k)] = v;
  }
}
// f += t2 of the last plane k' within b that holds a source (interior cells only)
__global__ void shift_k_add_kernel(const int8_t* t2, int8_t* f, LvlDims d, int b) {
  GRID_STRIDE(t, (long long)d.is * d.js * d.ks) {
    const int i = 1 + (int)(t % d.is), j = 1 + (int)((t / d.is) % d.js), kk = 1 + (int)(t / ((long long)d.is * d.js));
    int8_t v = 0;
    for (int k = min(kk + b, d.ks); k >= max(kk - b, 1); --k) {
      const int8_t x = t2[d.at(i, j, k)];
      if (x > 0) { v = x; break; }
    }
    int8_t& o = f[d.at(i, j, kk)];
    o = (int8_t)(o + v);
  }
}

__global__ void colate_kernel(int8_t* f, const int8_t* dom, LvlDims d) {
  GRID_STRIDE(t, (long long)d.is * d.js * d.ks) {
    const int i = 1 + (int)(t % d.is), j = 1 + (int)((t / d.is) % d.js), k = 1 + (int)(t / ((long long)d.is * d.js));
    const long long a = d.at(i, j, k);
    f[a] = f[a] < dom[a] ? f[a] : dom[a];
  }
}

// extend_borders with periodic directions, one direction per launch in the order x, y, z
// (a later direction reads ring cells an earlier one wrote): a periodic direction copies
// the far interior layer over its whole ring face (0..n+1 in the other two indices); a
// non-periodic one extends a 1 of the adjacent interior cell (other indices interior only)
__global__ void border_dir_kernel(int8_t* a, LvlDims d, int dir, int periodic) {
  const int e = periodic ? 2 : 0, o = periodic ? 0 : 1;
  const long long na = (dir == 0 ? d.js : d.is) + e, nb = (dir == 2 ? d.js : d.ks) + e;
  GRID_STRIDE(t, 2 * na * nb) {
    const bool hi = t >= na * nb;
    const long long r = hi ? t - na * nb : t;
    const int u = (int)(r % na) + o, v = (int)(r / na) + o;
    const int n = dir == 0 ? d.is : dir == 1 ? d.js : d.ks;
    const int ring = hi ? n + 1 : 0;
    const int src = periodic ? (hi ? 1 : n) : (hi ? n : 1);
    long long at, from;
    if (dir == 0) { at = d.at(ring, u, v); from = d.at(src, u, v); }
    else if (dir == 1) { at = d.at(u, ring, v); from = d.at(u, src, v); }
    else { at = d.at(u, v, ring); from = d.at(u, v, src); }
    if (periodic) a[at] = a[from];
    else if (a[from] == 1) a[at] = 1;
  }
}

// per: bit 0, 1, 2 set for periodic x, y, z; skip: leave the ring of periodic directions as it is
void borders(int8_t* a, LvlDims d, bool edges, cudaStream_t s, int per = 0, bool skip = false) {
  if (per == 0) {
    const long long n = 2LL * ((long long)d.js * d.ks + (long long)d.is * d.ks + (long long)d.is * d.js);
    extend_kernel<<<blocks_for(n, 256), 256, 0, s>>>(a, d);
  } else {
    for (int dir = 0; dir < 3; ++dir) {
      const bool p = (per >> dir) & 1;
      if (p && skip) continue;
      const long long na = (dir == 0 ? d.js : d.is) + (p ? 2 : 0), nb = (dir == 2 ? d.js : d.ks) + (p ? 2 : 0);
      border_dir_kernel<<<blocks_for(2 * na * nb, 256), 256, 0, s>>>(a, d, dir, p ? 1 : 0);
    }
  }
  if (edges) {
    edges_kernel<<<blocks_for(4LL * (d.is + d.js + d.ks), 256), 256, 0, s>>>(a, d);
    corners_kernel<<<1, 32, 0, s>>>(a, d);
  }
}

}  // namespace

void launch_domprep(int8_t* a, LvlDims d, const LvlBox* boxes, int nbox, cudaStream_t s, int per) {
  AMR_CUDA(cudaMemsetAsync(a, 0, d.size(), s));
  for (int b0 = 0; b0 < nbox; b0 += 65535)
    boxes_kernel<<<dim3(8, std::min(65535, nbox - b0)), 256, 0, s>>>(a, d, boxes + b0, std::min(65535, nbox - b0), 0);
  borders(a, d, true, s, per);
  AMR_CUDA(cudaGetLastError());
}

void launch_domshrink(const int8_t* in, int8_t* out, LvlDims d, cudaStream_t s, int per) {
  shrink_kernel<<<blocks_for(d.size(), 256), 256, 0, s>>>(in, out, d);
  borders(out, d, false, s, per, true);
  AMR_CUDA(cudaGetLastError());
}

void launch_domup(const int8_t* crse, LvlDims cd, int8_t* fine, LvlDims fd, int rx, int ry, int rz, cudaStream_t s, int per) {
  up_kernel<<<blocks_for(fd.size(), 256), 256, 0, s>>>(crse, cd, fine, fd, rx, ry, rz);
  borders(fine, fd, true, s, per);
  AMR_CUDA(cudaGetLastError());
}

void launch_domcopy_borders(int8_t* a, LvlDims d, cudaStream_t s, int per) {
  borders(a, d, false, s, per);
  AMR_CUDA(cudaGetLastError());
}

void launch_zero_interior(int8_t* f, LvlDims d, cudaStream_t s) {
  zero_interior_kernel<<<blocks_for((long long)d.is * d.js * d.ks, 256), 256, 0, s>>>(f, d);
  AMR_CUDA(cudaGetLastError());
}

void launch_flag_cells3(const void* pool, const PatchDev* patches, const int* plist, const long long* cell0, int np,
                        long long ncells, int flag_pressure, double gamma1, double tolsp, int nvar, int8_t* f, LvlDims d,
                        cudaStream_t s, bool f32) {
  if (ncells <= 0) return;
  if (f32)
    flag_cells_kernel<<<blocks_for(ncells, 256), 256, 0, s>>>(static_cast<const float*>(pool), patches, plist, cell0, np, ncells,
                                                              flag_pressure, gamma1, tolsp, nvar, f, d);
  else
    flag_cells_kernel<<<blocks_for(ncells, 256), 256, 0, s>>>(static_cast<const double*>(pool), patches, plist, cell0, np, ncells,
                                                              flag_pressure, gamma1, tolsp, nvar, f, d);
  AMR_CUDA(cudaGetLastError());
}

void launch_bufnst3(int8_t* f, LvlDims d, const LvlBox* proj, int nproj, int ibuff, int8_t* t1, int8_t* t2, cudaStream_t s) {
  for (int b0 = 0; b0 < nproj; b0 += 65535)
    boxes_kernel<<<dim3(8, std::min(65535, nproj - b0)), 256, 0, s>>>(f, d, proj + b0, std::min(65535, nproj - b0), 1);
  zero_ring_kernel<<<blocks_for(d.size(), 256), 256, 0, s>>>(f, d);
  shift_i_kernel<<<blocks_for((long long)(d.is + 2) * d.js * d.ks, 256), 256, 0, s>>>(f, t1, d, ibuff);
  shift_j_kernel<<<blocks_for((long long)(d.is + 2) * (d.js + 2) * d.ks, 256), 256, 0, s>>>(t1, t2, d, ibuff);
  shift_k_add_kernel<<<blocks_for((long long)d.is * d.js * d.ks, 256), 256, 0, s>>>(t2, f, d, ibuff);
  AMR_CUDA(cudaGetLastError());
}

void launch_colate3(int8_t* f, const int8_t* dom, LvlDims d, cudaStream_t s) {
  colate_kernel<<<blocks_for((long long)d.is * d.js * d.ks, 256), 256, 0, s>>>(f, dom, d);
  AMR_CUDA(cudaGetLastError());
}

// ======================================================================= signatures (signs.f)
namespace {
// The row / column / plane counts of the flagged cells (f != 0) of each box: blockIdx.y is
// the box, each warp takes i-rows (fixed j, k) of it in turn, 32 cells of a row at a time
// (lane = i, coalesced reads). The i-counts go to shared memory one lane per bin; the j-
// and k-counts of a chunk are summed across the warp first and added once. Counts are
// integers, so the order of the adds does not matter.
__global__ void signatures3_kernel(const int8_t* f, LvlDims d, const SigBox* boxes, const int* off, int* hist) {
  extern __shared__ int sh[];
  const SigBox B = boxes[blockIdx.y];
  const int ni = B.hi[0] - B.lo[0] + 1, nj = B.hi[1] - B.lo[1] + 1, nk = B.hi[2] - B.lo[2] + 1;
  const int nh = ni + nj + nk;
  for (int t = threadIdx.x; t < nh; t += blockDim.x) sh[t] = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const long long rows = (long long)nj * nk;
  for (long long r = (long long)blockIdx.x * nwarps + warp; r < rows; r += (long long)gridDim.x * nwarps) {
    const int j = (int)(r % nj), k = (int)(r / nj);
    const int8_t* row = f + d.at(B.lo[0], B.lo[1] + j, B.lo[2] + k);
    int cnt = 0;
    for (int i0 = 0; i0 < ni; i0 += 32) {
      const int i = i0 + lane;
      const int flag = (i < ni && row[i] != 0) ? 1 : 0;
      if (flag) atomicAdd(&sh[i], 1);
      cnt += __popc(__ballot_sync(0xffffffffu, flag));
    }
    if (lane == 0 && cnt) {
      atomicAdd(&sh[ni + j], cnt);
      atomicAdd(&sh[ni + nj + k], cnt);
    }
  }
  __syncthreads();
  int* h = hist + off[blockIdx.y];
  for (int t = threadIdx.x; t < nh; t += blockDim.x)
    if (sh[t]) atomicAdd(&h[t], sh[t]);
}
__global__ void scatter_points_kernel(const int* pts, int n, int8_t* f, LvlDims d) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x)
    f[d.at(pts[2 * t] + 1, pts[2 * t + 1] + 1, 1)] = 1;
}
}  // namespace

void launch_scatter_points2(const int* pts, int n, int8_t* f, LvlDims d, cudaStream_t s) {
  AMR_CUDA(cudaMemsetAsync(f, 0, (size_t)d.size(), s));
  if (n > 0) scatter_points_kernel<<<blocks_for(n, 256), 256, 0, s>>>(pts, n, f, d);
  AMR_CUDA(cudaGetLastError());
}

void launch_signatures3(const int8_t* f, LvlDims d, const SigBox* boxes, int nbox, const int* off, int total, int maxlen,
                        long long maxrows, int* hist, cudaStream_t s) {
  if (nbox <= 0) return;
  AMR_CUDA(cudaMemsetAsync(hist, 0, sizeof(int) * (size_t)total, s));
  // blocks of 8 warps, a warp per i-row: enough blocks per box for its rows
  const int slabs = (int)std::max<long long>(1, std::min<long long>(64, (maxrows + 7) / 8));
  for (int base = 0; base < nbox; base += 65535) {
    const int cnt = std::min(65535, nbox - base);
    signatures3_kernel<<<dim3(slabs, cnt), 256, sizeof(int) * (size_t)maxlen, s>>>(f, d, boxes + base, off + base, hist);
  }
  AMR_CUDA(cudaGetLastError());
}

// ======================================================================= Richardson estimation
namespace {
template <class T>
__global__ void coarsen3_kernel(T* pool, const Rect3* rects, const int* rect_of, const PatchDev* vp, int nvar) {
  const int k = blockIdx.y;
  const PatchDev P = vp[k];
  const Rect3 R = rects[rect_of[k]];
  const T* src = pool + R.off;
  T* dst = pool + P.q[0];
  const long long sj = R.ni, sk = (long long)R.ni * R.nj, splane = sk * R.nk;
  const long long n = (long long)P.mitot * P.mjtot * P.mktot;
  GRID_STRIDE(t, n * nvar) {
    const int m = (int)(t / n);
    const long long rem = t % n;
    const int i = (int)(rem % P.mitot), j = (int)((rem / P.mitot) % P.mjtot), kk = (int)(rem / ((long long)P.mitot * P.mjtot));
    const T* s0 = src + m * splane + (2 * kk) * sk + (2 * j) * sj + 2 * i;
    const double v = (((((((double)s0[0] + (double)s0[1]) + (double)s0[sj]) + (double)s0[sj + 1]) + (double)s0[sk]) + (double)s0[sk + 1]) +
                      (double)s0[sk + sj]) + (double)s0[sk + sj + 1];
    dst[m * n + rem] = (T)(v / 8.0);
  }
}
template <class T>
__global__ void errf3_kernel(const T* pool, const PatchDev* vp, int np, double order, double tol, int8_t* f, LvlDims d) {
  const int k = blockIdx.y;
  const PatchDev C = vp[k], F = vp[np + k];
  const int nxc = (F.ihi - F.ilo + 1) / 2, nyc = (F.jhi - F.jlo + 1) / 2, nzc = (F.khi - F.klo + 1) / 2;
  const T* fine = pool + F.q[1];
  const T* crse = pool + C.q[1];
  const long long fj = F.mitot, fk = (long long)F.mitot * F.mjtot;
  GRID_STRIDE(t, (long long)nxc * nyc * nzc) {
    const int ic = (int)(t % nxc), jc = (int)((t / nxc) % nyc), kc = (int)(t / ((long long)nxc * nyc));
    const T* f0 = fine + (2 * kc + NGF) * fk + (2 * jc + NGF) * fj + (2 * ic + NGF);
    // errf1.f: term1..term8 in the reference's order
    const double aval = ((((((((double)f0[0] + (double)f0[1]) + (double)f0[fj + 1]) + (double)f0[fj]) + (double)f0[fk]) + (double)f0[fk + 1]) +
                         (double)f0[fk + fj + 1]) + (double)f0[fk + fj]) / 8.0;
    const double c = (double)crse[((long long)(kc + NGF) * C.mjtot + (jc + NGF)) * C.mitot + (ic + NGF)];
    const double est = fabs((aval - c) / order);
    if (est >= tol) {
      const int gi = F.ilo + 2 * ic + 1, gj = F.jlo + 2 * jc + 1, gk = F.klo + 2 * kc + 1;  // array index = global + 1
      for (int dk = 0; dk <= 1; ++dk)
        for (int dj = 0; dj <= 1; ++dj)
          for (int di = 0; di <= 1; ++di) {
            int8_t& a = f[d.at(gi + di, gj + dj, gk + dk)];
            a = (int8_t)(a + 2);
          }
    }
  }
}
}  // namespace

void launch_coarsen3(void* pool, const Rect3* rects, const int* rect_of, const PatchDev* vp, int np, int nvar, cudaStream_t s,
                     bool f32) {
  for (int base = 0; base < np; base += 65535) {
    const int n = std::min(65535, np - base);
    if (f32) coarsen3_kernel<<<dim3(16, n), 256, 0, s>>>(static_cast<float*>(pool), rects, rect_of + base, vp + base, nvar);
    else coarsen3_kernel<<<dim3(16, n), 256, 0, s>>>(static_cast<double*>(pool), rects, rect_of + base, vp + base, nvar);
    AMR_CUDA(cudaGetLastError());
  }
}
void launch_errf3(const void* pool, const PatchDev* vp, int np, double order, double tol, int8_t* f, LvlDims d, cudaStream_t s,
                  bool f32) {
  for (int base = 0; base < np; base += 65535) {
    const int n = std::min(65535, np - base);
    // the partners of vp[base..] are np entries further on, from the shifted pointer too
    if (f32) errf3_kernel<<<dim3(8, n), 256, 0, s>>>(static_cast<const float*>(pool), vp + base, np, order, tol, f, d);
    else errf3_kernel<<<dim3(8, n), 256, 0, s>>>(static_cast<const double*>(pool), vp + base, np, order, tol, f, d);
    AMR_CUDA(cudaGetLastError());
  }
}

}  // namespace amrb
