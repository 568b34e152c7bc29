// HEALPix neighbour table and the neighbour-average steps of the reference's
// inpainting (polyspec/weighting.py:87-146), FP64.
//
//  * ps_healpix_neighbours: out[p][k], k = SW, W, NW, N, NE, E, SE, S, the RING
//    neighbours of every pixel (healpy.get_all_neighbours, which the reference
//    calls).  One thread per face pixel (f, x, y): the in-face neighbours are
//    (x + dx, y + dy); one outside the face is wrapped modulo Nside into the face of
//    its 3 x 3 cell and mapped by that cell's lattice symmetry (flip x, flip y,
//    swap, in that order), both from a 2 x 9 x 12 table the host derives from the
//    faces' shared vertices; -1 where the cell has no face (three faces meet).
//    RING indices from face coordinates: ring jr = jrll Nside - x - y - 1 and
//    azimuth jp = (jpll nr + x - y + 1 + s) / 2 in the ring's numbering (Gorski et
//    al. 2005, with s the equatorial rings' half-pixel shift).
//  * ps_inpaint_average: dst[p] = the average of src over the 8 neighbours of p
//    for each p in a list, as np.average(this_map[neighbors], axis=0) (plain mean,
//    neighbours added in order, divided by 8) or, with weighted = 1, as the fill
//    step's np.average(..., weights=this_map[neighbors] != 1e-30); a neighbour -1
//    reads the last pixel, as numpy's index -1 does.  dst is a separate buffer, so
//    every update of a pass reads the values from before the pass.
#include "ps_common.cuh"
#include "ps_stats.cuh"

namespace ps {
namespace {

__constant__ int c_jrll[12] = {2, 2, 2, 2, 3, 3, 3, 3, 4, 4, 4, 4};
__constant__ int c_jpll[12] = {1, 3, 5, 7, 0, 2, 4, 6, 1, 3, 5, 7};

__device__ int64_t xyf2ring(int64_t n, int f, int64_t x, int64_t y) {
  const int64_t npix = 12 * n * n, ncap = 2 * n * (n - 1);
  const int64_t jr = c_jrll[f] * n - x - y - 1;
  int64_t nr, nbefore, kshift = 0;
  if (jr < n) {
    nr = jr;
    nbefore = 2 * nr * (nr - 1);
  } else if (jr > 3 * n) {
    nr = 4 * n - jr;
    nbefore = npix - 2 * (nr + 1) * nr;
  } else {
    nr = n;
    nbefore = ncap + (jr - n) * 4 * n;
    kshift = (jr - n) & 1;
  }
  int64_t jp = (c_jpll[f] * nr + x - y + 1 + kshift) / 2;
  if (jp > 4 * nr) jp -= 4 * nr;
  if (jp < 1) jp += 4 * nr;
  return nbefore + jp - 1;
}

__global__ void neighbours_kernel(int n, const int* __restrict__ tab, int* __restrict__ out) {
  const int64_t total = 12 * int64_t(n) * n;
  const int dxs[8] = {-1, -1, 0, 1, 1, 1, 0, -1};
  const int dys[8] = {0, 1, 1, 1, 0, -1, -1, -1};
  for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < total; t += int64_t(gridDim.x) * blockDim.x) {
    const int f = int(t / (int64_t(n) * n));
    const int64_t rem = t % (int64_t(n) * n);
    const int64_t y = rem / n, x = rem % n;
    const int64_t p = xyf2ring(n, f, x, y);
    for (int k = 0; k < 8; ++k) {
      int64_t X = x + dxs[k], Y = y + dys[k];
      int64_t q;
      if (X >= 0 && X < n && Y >= 0 && Y < n) {
        q = xyf2ring(n, f, X, Y);
      } else {
        const int cell = (X < 0 ? 0 : X >= n ? 2 : 1) + 3 * (Y < 0 ? 0 : Y >= n ? 2 : 1);
        const int g = __ldg(tab + cell * 12 + f), bits = __ldg(tab + 108 + cell * 12 + f);
        if (g < 0) {
          q = -1;
        } else {
          X = (X + n) % n;
          Y = (Y + n) % n;
          if (bits & 1) X = n - 1 - X;
          if (bits & 2) Y = n - 1 - Y;
          if (bits & 4) {
            const int64_t s = X;
            X = Y;
            Y = s;
          }
          q = xyf2ring(n, g, X, Y);
        }
      }
      out[p * 8 + k] = int(q);
    }
  }
}

__global__ void inpaint_average_kernel(const double* __restrict__ src, const int* __restrict__ pix, int64_t n,
                                       const int* __restrict__ nb, int64_t npix, int weighted,
                                       double* __restrict__ dst) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    const int64_t p = __ldg(pix + i);
    double s = 0.0, ws = 0.0;
    for (int k = 0; k < 8; ++k) {
      int64_t q = __ldg(nb + p * 8 + k);
      if (q < 0) q = npix - 1;
      const double v = __ldg(src + q);
      if (weighted) {
        const double w = (v != 1e-30) ? 1.0 : 0.0;
        s += v * w;
        ws += w;
      } else {
        s += v;
      }
    }
    dst[p] = weighted ? s / ws : s / 8.0;
  }
}

}  // namespace
}  // namespace ps

using namespace ps;

extern "C" int ps_healpix_neighbours(int nside, const int* tables, int* out, cudaStream_t stream) {
  if (nside <= 0 || nside > 8192 || !tables || !out) return PS_ERR_INVALID;
  const int64_t total = 12 * int64_t(nside) * nside;
  StatScope sc(PS_K_PIXEL, 0.0, 32.0 * double(total), stream);
  int64_t g = (total + 255) / 256;
  if (g > 148 * 16) g = 148 * 16;
  neighbours_kernel<<<int(g), 256, 0, stream>>>(nside, tables, out);
  PS_LAUNCH_CHECK();
  return PS_OK;
}

extern "C" int ps_inpaint_average(const double* src, const int* pix, int64_t n, const int* nb, int64_t npix,
                                  int weighted, double* dst, cudaStream_t stream) {
  if (!src || !nb || !dst || n < 0 || npix <= 0 || (n > 0 && !pix) || src == dst) return PS_ERR_INVALID;
  if (n == 0) return PS_OK;
  StatScope sc(PS_K_PIXEL, 0.0, 80.0 * double(n), stream);
  int64_t g = (n + 255) / 256;
  if (g > 148 * 16) g = 148 * 16;
  inpaint_average_kernel<<<int(g), 256, 0, stream>>>(src, pix, n, nb, npix, weighted ? 1 : 0, dst);
  PS_LAUNCH_CHECK();
  return PS_OK;
}
