// Ghost-fill executor whose coarse scratch lives in a fixed device array.
//
// The fill programs of a level (bound.f90 / filpatch.f90 / saveqc.f) stage
// coarse values in scratch rectangles before interpolating from them. The
// regular executor (kernels2d.cu) takes those rectangles from the context's
// device pool, which grows at regrid time. The kernels here run the same
// programs with every rectangle placed in `g_fill_scratch`, a file-scope device
// array of fixed size, so a level substep can run without any device
// allocation. A program whose scratch exceeds the array is rejected on the host.
#include "kernels2d.cuh"
#include "noalloc2d.cuh"

#include <mutex>

namespace amrb {

static __device__ __align__(256) double g_fill_scratch[NOALLOC_SCRATCH_DOUBLES];

namespace {

__device__ __forceinline__ int floordiv_na(int a, int b) { return (a >= 0) ? a / b : -((-a + b - 1) / b); }

// Scratch rect r of the program, placed in the fixed array.
__device__ __forceinline__ double* rect_base(const FillArgs& a, const double* scratch, long long off0, int r) {
  return const_cast<double*>(scratch) + (a.rects[r].off - off0);
}

__global__ void fill_kernel_fixed(FillArgs a, const double* scratch, long long off0) {
  const int c = blockIdx.x;
  if (c >= a.nchunks) return;
  const FillChunk ch = a.chunks[c];
  if ((int)threadIdx.x >= ch.count) return;
  const FillOp o = a.ops[ch.op];
  const int cell = ch.start + threadIdx.x;
  const int ia = cell % o.ni, jb = cell / o.ni;
  const int nvar = a.nvar;
  if (o.kind == FILL_RING) {
    // cstore.f:4-63: ring of coarse values around a fine grid into qc1d of the kid
    const ScratchRect& R = a.rects[o.src];
    const int nrow = R.ni, ncol = R.nj;
    int k = cell, ii, jj;
    if (k < ncol - 2) { ii = 0; jj = 1 + k; }
    else if ((k -= ncol - 2) < nrow - 2) { ii = 1 + k; jj = ncol - 1; }
    else if ((k -= nrow - 2) < ncol - 2) { ii = nrow - 1; jj = 1 + k; }
    else { k -= ncol - 2; ii = 1 + k; jj = 0; }
    const PatchDev& K = a.patches[o.dst_patch];
    double* qc1d = a.regs + K.ffl + (long long)nvar * K.lenbc + (long long)nvar * cell;
    const double* src = rect_base(a, scratch, off0, o.src);
    const long long pl = (long long)nrow * ncol;
    for (int m = 0; m < nvar; ++m) qc1d[m] = src[m * pl + (long long)jj * nrow + ii];
    return;
  }
  int ldi; long long plane; double* dst;
  if (o.dst_patch >= 0) {
    const PatchDev& P = a.patches[o.dst_patch];
    ldi = P.mitot; plane = (long long)P.mitot * P.mjtot;
    dst = static_cast<double*>(a.pool) + P.q[P.cur];
  } else {
    const ScratchRect& R = a.rects[o.dst_rect];
    ldi = R.ni; plane = (long long)R.ni * R.nj;
    dst = rect_base(a, scratch, off0, o.dst_rect);
  }
  const long long dk = (long long)(o.dj0 + jb) * ldi + (o.di0 + ia);
  if (o.kind == FILL_COPY) {
    const PatchDev& S = a.patches[o.src];
    const long long sp = (long long)S.mitot * S.mjtot;
    const long long sk = (long long)(o.sj0 + jb) * S.mitot + (o.si0 + ia);
    int mode = 0; double ai = 1.0, ac = 0.0;
    if (o.level >= 0) { mode = a.modes.mode[o.level]; ai = a.modes.alphai[o.level]; ac = a.modes.alphac[o.level]; }
    const double* qn = static_cast<double*>(a.pool) + S.q[S.cur];
    const double* qo = static_cast<double*>(a.pool) + S.q[1 - S.cur];
    for (int m = 0; m < nvar; ++m) {
      double v;
      if (mode == 0) v = qn[m * sp + sk];
      else if (mode == 1) v = qo[m * sp + sk];
      else v = qn[m * sp + sk] * ai + qo[m * sp + sk] * ac;
      dst[m * plane + dk] = v;
    }
    return;
  }
  const ScratchRect& R = a.rects[o.src];
  const double* vc = rect_base(a, scratch, off0, o.src);
  if (o.kind == FILL_PIECE) {
    const long long sp = (long long)R.ni * R.nj;
    const long long sk = (long long)(o.sj0 + jb) * R.ni + (o.si0 + ia);
    for (int m = 0; m < nvar; ++m) dst[m * plane + dk] = vc[m * sp + sk];
    return;
  }
  const long long cp = (long long)R.ni * R.nj;
  const int lev = o.level;
  const int rx = a.lc.intratx[lev - 1], ry = a.lc.intraty[lev - 1];
  const int ifg = o.si0 + ia, jfg = o.sj0 + jb;
  if (o.kind == FILL_INTERP) {
    // filpatch.f90:259-327 limited interpolation from the coarse scratch rect
    const double dxf = a.lc.hx[lev], dyf = a.lc.hy[lev], dxc = a.lc.hx[lev - 1], dyc = a.lc.hy[lev - 1];
    const int icg = floordiv_na(ifg, rx), jcg = floordiv_na(jfg, ry);
    const int ic = icg - o.cilo + 1, jc = jcg - o.cjlo + 1;
    const double xlow_c = a.xlower + o.cilo * dxc, ylow_c = a.ylower + o.cjlo * dyc;
    const double ycc = ylow_c + (jc - 0.5) * dyc;
    const double ycf = a.ylower + (jfg + 0.5) * dyf;
    const double eta2 = (ycf - ycc) / dyc;
    const double xcc = xlow_c + (ic - 0.5) * dxc;
    const double xcf = a.xlower + (ifg + 0.5) * dxf;
    const double eta1 = (xcf - xcc) / dxc;
    auto CI = [&](int m, int i, int j) { return vc[m * cp + (long long)(j - 1) * R.ni + (i - 1)]; };
    for (int m = 0; m < nvar; ++m) {
      const double valp10 = CI(m, ic + 1, jc), valm10 = CI(m, ic - 1, jc), valc = CI(m, ic, jc);
      const double valp01 = CI(m, ic, jc + 1), valm01 = CI(m, ic, jc - 1);
      const double dupc = valp10 - valc, dumc = valc - valm10, ducc = valp10 - valm10;
      double du = dmin(fabs(dupc), fabs(dumc));
      du = dmin(2.0 * du, 0.5 * fabs(ducc));
      const double fu = dmax(0.0, dsign(1.0, dupc * dumc));
      const double uslope = du * dsign(1.0, ducc) * fu;
      const double dvpc = valp01 - valc, dvmc = valc - valm01, dvcc = valp01 - valm01;
      double dv = dmin(fabs(dvpc), fabs(dvmc));
      dv = dmin(2.0 * dv, 0.5 * fabs(dvcc));
      const double fv = dmax(0.0, dsign(1.0, dvpc * dvmc));
      const double vslope = dv * dsign(1.0, dvcc) * fv;
      dst[m * plane + dk] = valc + eta1 * uslope + eta2 * vslope;
    }
    return;
  }
  if (o.kind == FILL_FILVAL) {
    // filval.f90:150-185 minmod-limited interpolation into an uncovered new-grid cell
    const int icg = floordiv_na(ifg, rx), jcg = floordiv_na(jfg, ry);
    const int ico = ifg - icg * rx + 1, jco = jfg - jcg * ry + 1;
    const int i = icg - o.cilo + 1, j = jcg - o.cjlo + 1;
    auto VC = [&](int m, int ii, int jj) { return vc[m * cp + (long long)(jj - 1) * R.ni + (ii - 1)]; };
    const double yoff = ((double)jco - 0.5) / ry - 0.5;
    const double xoff = ((double)ico - 0.5) / rx - 0.5;
    for (int m = 0; m < nvar; ++m) {
      double s1p = VC(m, i + 1, j) - VC(m, i, j), s1m = VC(m, i, j) - VC(m, i - 1, j);
      double slopex = dmin(fabs(s1p), fabs(s1m)) * dsign(1.0, VC(m, i + 1, j) - VC(m, i - 1, j));
      if (s1m * s1p <= 0.0) slopex = 0.0;
      s1p = VC(m, i, j + 1) - VC(m, i, j); s1m = VC(m, i, j) - VC(m, i, j - 1);
      double slopey = dmin(fabs(s1p), fabs(s1m)) * dsign(1.0, VC(m, i, j + 1) - VC(m, i, j - 1));
      if (s1m * s1p <= 0.0) slopey = 0.0;
      dst[m * plane + dk] = VC(m, i, j) + xoff * slopex + yoff * slopey;
    }
  }
}

// bc2amr.f90:84-297 on a patch or on a fixed-scratch rect. phase 0: x sides; 1: y sides.
__global__ void bc_kernel_fixed(BcArgs a, int phase, const double* scratch, long long off0) {
  const int op = blockIdx.y;
  if (op >= a.nops) return;
  const BcOp o = a.ops[op];
  double* v; const int nrow = o.nrow, ncol = o.ncol;
  if (o.dst_patch >= 0) { const PatchDev& P = a.patches[o.dst_patch]; v = static_cast<double*>(a.pool) + P.q[P.cur]; }
  else v = const_cast<double*>(scratch) + (a.rects[o.dst_rect].off - off0);
  const long long plane = (long long)nrow * ncol;
  auto V = [&](int m, int i, int j) -> double& { return v[m * plane + (long long)(j - 1) * nrow + (i - 1)]; };
  const int nvar = a.nvar;
  if (phase == 0) {
    const int nl = (o.nxl > 0 && (o.bxl == 1 || o.bxl == 3)) ? o.nxl : 0;
    const int nr = (o.ibeg > 0 && (o.bxr == 1 || o.bxr == 3)) ? nrow - o.ibeg + 1 : 0;
    const int tot = (nl + nr) * ncol;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < tot; t += gridDim.x * blockDim.x) {
      const int j = t / (nl + nr) + 1, k = t % (nl + nr);
      if (k < nl) {
        const int i = k + 1;
        const int src = (o.bxl == 1) ? o.nxl + 1 : 2 * o.nxl + 1 - i;
        for (int m = 0; m < nvar; ++m) V(m, i, j) = V(m, src, j);
        if (o.bxl == 3) V(1, i, j) = -V(1, i, j);
      } else {
        const int i = o.ibeg + (k - nl);
        const int src = (o.bxr == 1) ? o.ibeg - 1 : 2 * o.ibeg - 1 - i;
        for (int m = 0; m < nvar; ++m) V(m, i, j) = V(m, src, j);
        if (o.bxr == 3) V(1, i, j) = -V(1, i, j);
      }
    }
  } else {
    const int nb = (o.nyb > 0 && (o.byl == 1 || o.byl == 3)) ? o.nyb : 0;
    const int nt = (o.jbeg > 0 && (o.byr == 1 || o.byr == 3)) ? ncol - o.jbeg + 1 : 0;
    const int tot = (nb + nt) * nrow;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < tot; t += gridDim.x * blockDim.x) {
      const int i = t % nrow + 1, k = t / nrow;
      if (k < nb) {
        const int j = k + 1;
        const int src = (o.byl == 1) ? o.nyb + 1 : 2 * o.nyb + 1 - j;
        for (int m = 0; m < nvar; ++m) V(m, i, j) = V(m, i, src);
        if (o.byl == 3) V(2, i, j) = -V(2, i, j);
      } else {
        const int j = o.jbeg + (k - nb);
        const int src = (o.byr == 1) ? o.jbeg - 1 : 2 * o.jbeg - 1 - j;
        for (int m = 0; m < nvar; ++m) V(m, i, j) = V(m, i, src);
        if (o.byr == 3) V(2, i, j) = -V(2, i, j);
      }
    }
  }
}

std::mutex g_sym_mu;
double* g_sym_addr[64] = {nullptr};

}  // namespace

int fixed_scratch_address(double** out, std::string& err) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) { err = std::string("cudaGetDevice: ") + cudaGetErrorString(e); return 1; }
  if (dev < 0 || dev >= 64) { err = "device ordinal out of range for the fixed scratch table"; return 1; }
  std::lock_guard<std::mutex> g(g_sym_mu);
  if (!g_sym_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_fill_scratch);
    if (e != cudaSuccess) { err = std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e); return 1; }
    g_sym_addr[dev] = static_cast<double*>(p);
  }
  *out = g_sym_addr[dev];
  return 0;
}

void launch_fill_fixed(const FillArgs& a, const double* scratch, long long off0, cudaStream_t s) {
  if (a.nchunks <= 0) return;
  fill_kernel_fixed<<<a.nchunks, 128, 0, s>>>(a, scratch, off0);
  AMR_CUDA(cudaGetLastError());
}

void launch_bc_fixed(const BcArgs& a, int phase, const double* scratch, long long off0, cudaStream_t s) {
  if (a.nops <= 0) return;
  for (int base = 0; base < a.nops; base += 65535) {
    BcArgs b = a;
    b.ops = a.ops + base;
    b.nops = std::min(65535, a.nops - base);
    dim3 grid(2, b.nops);
    bc_kernel_fixed<<<grid, 128, 0, s>>>(b, phase, scratch, off0);
    AMR_CUDA(cudaGetLastError());
  }
}

}  // namespace amrb
