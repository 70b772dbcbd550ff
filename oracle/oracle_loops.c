/*
 * ORACLE — test infrastructure only.  Plain-C FP64 restatement of the reference's
 * O(N_bins * N^3) real-space grid loops, used as the checker for the CUDA path and as
 * the CPU baseline.  Never linked into the product.
 *
 *   oracle_triplet_sum  <- assemble_b3   PolyBin3D/cython/utils.pyx:614-636
 *                          sum_triplet   PolyBin3D/cython/utils.pyx:357-366
 *   oracle_pair_sum     <- sum_pair      PolyBin3D/cython/utils.pyx:343-352
 *
 * Maps are C-contiguous float64 arrays of n_vox voxels each.  For each triplet t the
 * sum  out[t] = sum_x A[i1[t]](x) * B[i2[t]](x) * C[i3[t]](x)  runs in the reference's
 * voxel order (i1,i2,i3 loops = linear order), one OpenMP task per triplet as the
 * reference's prange over bins (utils.pyx:621).
 */
#include <stdint.h>
#include <stddef.h>

void oracle_triplet_sum(const double *A, const double *B, const double *C,
                        int64_t n_vox, const int64_t *idx, int64_t n_trip,
                        double *out, int nthreads)
{
#pragma omp parallel for schedule(static) num_threads(nthreads)
    for (int64_t t = 0; t < n_trip; ++t) {
        const double *a = A + idx[3 * t + 0] * n_vox;
        const double *b = B + idx[3 * t + 1] * n_vox;
        const double *c = C + idx[3 * t + 2] * n_vox;
        double acc = 0.0;
        for (int64_t x = 0; x < n_vox; ++x) acc += a[x] * b[x] * c[x];
        out[t] = acc;
    }
}

void oracle_pair_sum(const double *A, const double *B, int64_t n_vox,
                     const int64_t *idx, int64_t n_pair, double *out, int nthreads)
{
#pragma omp parallel for schedule(static) num_threads(nthreads)
    for (int64_t t = 0; t < n_pair; ++t) {
        const double *a = A + idx[2 * t + 0] * n_vox;
        const double *b = B + idx[2 * t + 1] * n_vox;
        double acc = 0.0;
        for (int64_t x = 0; x < n_vox; ++x) acc += a[x] * b[x];
        out[t] = acc;
    }
}
