// Gaussian smoothing of the summed velocity gradient (ExtraParams.smoothgradkern = l > 0):
// smoothgradient, gaussian_kernel and smoothimg of src/EikSolv/utils.jl:22-96, applied to
// the group-summed gradient before it is returned (src/EikSolv/eikmaingrad.jl:144-147).
//
// What the reference computes: it pads the gradient with zeros (l÷2 nodes before and
// l÷2+1 after the data on every axis), correlates the padded array with the l^d Gaussian
// kernel at every node whose index is at least l÷2+1 from both ends, and crops the data
// back out. Every node of the original grid is such an interior node, so the result is the
// zero-padded correlation
//     out[p] = Σ_J in[p + J] · K[J],   J ∈ [-l÷2, l÷2]^d,
// accumulated from 0.0 with J in column-major order (first axis fastest, as Julia's
// CartesianIndices iterate). A term on the padding adds +0.0 to a partial sum that is never
// -0.0 (it starts at +0.0 and an exact cancellation rounds to +0.0), so reading a
// zero-filled halo, or skipping the term, leaves every bit of the sum as the reference's.
//
// Kernel weights: K[J] = exp(-r²/(2s)) / Σ, r = sqrt(Σ_a J_a²), s = l/2 - sqrt(l/2),
// evaluated on the host in double precision in the reference's order (utils.jl:19-35).
//
// Layout: one CTA of 256 threads per output tile (2D 32×8, 3D 32×4×2 nodes, x fastest so
// every row of a warp is one coalesced 256-byte segment). The tile plus its halo of l÷2 on
// each side is staged in shared memory once (zeros outside the grid); each thread then
// sums its l^d products from shared memory, the weight of each step being one broadcast
// load. When the staged tile would not fit in shared memory (3D with l > 21) the kernel
// reads the input straight from global memory through the read-only cache instead.
// Cost: 16 B of HBM traffic per node (read once, write once) and 2·l^d FP64 operations per
// node, so it is HBM-bound for small l and FP64-bound for large l.
#include <cuda_runtime.h>

#include <cmath>
#include <vector>

#include "kernels.cuh"

namespace eik {

constexpr int SM_THREADS = 256;

template <int ND>
struct SmoothTile {
  static constexpr int X = 32, Y = 8 / (ND == 3 ? 2 : 1), Z = ND == 3 ? 2 : 1;
};

struct SmoothArgs {
  const double* in;
  double* out;
  const double* w;  // l^ND weights, first axis fastest
  int n[3];
  int l, half;
  long long tiles[3];  // tiles per axis
};

// Staged variant: the tile's input box (tile + halo) is copied to shared memory first.
template <int ND>
__global__ void __launch_bounds__(SM_THREADS) smooth_tiled_kernel(SmoothArgs a) {
  extern __shared__ double box[];
  using T = SmoothTile<ND>;
  const long long b = blockIdx.x;
  const long long tx = b % a.tiles[0], ty = (b / a.tiles[0]) % a.tiles[1], tz = b / (a.tiles[0] * a.tiles[1]);
  const int x0 = (int)tx * T::X, y0 = (int)ty * T::Y, z0 = (int)tz * T::Z;
  const int l = a.l, h = a.half;
  const int bx = T::X + l - 1, by = T::Y + l - 1, bz = ND == 3 ? T::Z + l - 1 : 1;
  const int nbox = bx * by * bz;
  for (int q = threadIdx.x; q < nbox; q += SM_THREADS) {
    const int qx = q % bx, qy = (q / bx) % by, qz = q / (bx * by);
    const int gx = x0 - h + qx, gy = y0 - h + qy, gz = ND == 3 ? z0 - h + qz : 0;
    double v = 0.0;
    if (gx >= 0 && gx < a.n[0] && gy >= 0 && gy < a.n[1] && gz >= 0 && gz < a.n[2])
      v = __ldg(a.in + (long long)gx + (long long)a.n[0] * ((long long)gy + (long long)a.n[1] * gz));
    box[q] = v;
  }
  __syncthreads();
  const int ix = threadIdx.x % T::X, iy = (threadIdx.x / T::X) % T::Y, iz = threadIdx.x / (T::X * T::Y);
  const int px = x0 + ix, py = y0 + iy, pz = z0 + iz;
  if (px >= a.n[0] || py >= a.n[1] || pz >= a.n[2]) return;
  double acc = 0.0;
  int kq = 0;
  for (int kz = 0; kz < (ND == 3 ? l : 1); kz++)
    for (int ky = 0; ky < l; ky++) {
      const double* row = box + ix + bx * ((iy + ky) + by * (iz + kz));
      for (int kx = 0; kx < l; kx++, kq++) acc = acc + row[kx] * __ldg(a.w + kq);
    }
  a.out[(long long)px + (long long)a.n[0] * ((long long)py + (long long)a.n[1] * pz)] = acc;
}

// Unstaged variant for kernels too wide to stage: terms outside the grid are skipped.
template <int ND>
__global__ void __launch_bounds__(SM_THREADS) smooth_direct_kernel(SmoothArgs a) {
  using T = SmoothTile<ND>;
  const long long b = blockIdx.x;
  const long long tx = b % a.tiles[0], ty = (b / a.tiles[0]) % a.tiles[1], tz = b / (a.tiles[0] * a.tiles[1]);
  const int px = (int)tx * T::X + threadIdx.x % T::X;
  const int py = (int)ty * T::Y + (threadIdx.x / T::X) % T::Y;
  const int pz = (int)tz * T::Z + threadIdx.x / (T::X * T::Y);
  if (px >= a.n[0] || py >= a.n[1] || pz >= a.n[2]) return;
  const int l = a.l, h = a.half;
  double acc = 0.0;
  int kq = 0;
  for (int kz = 0; kz < (ND == 3 ? l : 1); kz++) {
    const int gz = ND == 3 ? pz + kz - h : 0;
    for (int ky = 0; ky < l; ky++) {
      const int gy = py + ky - h;
      const bool rowin = gz >= 0 && gz < a.n[2] && gy >= 0 && gy < a.n[1];
      const double* row = a.in + (long long)a.n[0] * ((long long)gy + (long long)a.n[1] * gz);
      for (int kx = 0; kx < l; kx++, kq++) {
        const int gx = px + kx - h;
        if (rowin && gx >= 0 && gx < a.n[0]) acc = acc + __ldg(row + gx) * __ldg(a.w + kq);
      }
    }
  }
  a.out[(long long)px + (long long)a.n[0] * ((long long)py + (long long)a.n[1] * pz)] = acc;
}

template <int ND>
static cudaError_t launch_nd(SmoothArgs a, cudaStream_t st) {
  using T = SmoothTile<ND>;
  a.tiles[0] = (a.n[0] + T::X - 1) / T::X;
  a.tiles[1] = (a.n[1] + T::Y - 1) / T::Y;
  a.tiles[2] = (a.n[2] + T::Z - 1) / T::Z;
  const long long nblk = a.tiles[0] * a.tiles[1] * a.tiles[2];
  if (nblk > 0x7fffffffLL) return cudaErrorInvalidValue;
  const long long bz = ND == 3 ? T::Z + a.l - 1 : 1;
  const size_t smem = sizeof(double) * (size_t)((T::X + a.l - 1) * (long long)(T::Y + a.l - 1) * bz);
  int dev = 0, optin = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if (smem <= (size_t)optin) {
    cudaError_t e = cudaFuncSetAttribute(smooth_tiled_kernel<ND>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    smooth_tiled_kernel<ND><<<(unsigned)nblk, SM_THREADS, smem, st>>>(a);
  } else {
    smooth_direct_kernel<ND><<<(unsigned)nblk, SM_THREADS, 0, st>>>(a);
  }
  return cudaGetLastError();
}

// gaussian_kernel(dim, l) of utils.jl:19-35, normalised, first axis fastest.
std::vector<double> gaussian_weights(int l, int dim) {
  long long kn = 1;
  for (int d = 0; d < dim; d++) kn *= l;
  std::vector<double> w((size_t)kn);
  const double s = ((double)l / 2.0) - std::sqrt((double)l / 2.0);
  for (long long q = 0; q < kn; q++) {
    long long rr = 0, t = q;
    for (int d = 0; d < dim; d++) {
      const long long pos = t % l + 1 - (l / 2 + 1);
      t /= l;
      rr += pos * pos;
    }
    const double r = std::sqrt((double)rr);
    w[(size_t)q] = std::exp(-(r * r) / (2.0 * s));
  }
  double sum = 0.0;
  for (long long q = 0; q < kn; q++) sum += w[(size_t)q];
  for (long long q = 0; q < kn; q++) w[(size_t)q] = w[(size_t)q] / sum;
  return w;
}

cudaError_t launch_smoothgrad(const GridDesc& g, int l, const double* d_w, const double* in, double* out,
                              cudaStream_t st) {
  SmoothArgs a;
  a.in = in;
  a.out = out;
  a.w = d_w;
  a.n[0] = g.n[0];
  a.n[1] = g.n[1];
  a.n[2] = g.nd == 3 ? g.n[2] : 1;
  a.l = l;
  a.half = l / 2;
  return g.nd == 3 ? launch_nd<3>(a, st) : launch_nd<2>(a, st);
}

}  // namespace eik
