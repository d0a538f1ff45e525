// Spin-summed active densities for the orbital optimiser (sm_100a).
//
// hilbert's PackSpatialDensity (src/v2rdm_casscf/v2rdm_solver.cc:3110-3219,
// C1) loops over geminal pairs (ij, kl), forms a value from up to 16 D2
// elements and stores it at the packed index INDEX(INDEX(i,k), INDEX(j,l)).
// Eight (i, j, k, l) reach each packed index; the loop's last one (the
// largest ij * gab + kl) is the value that stays.  Here one thread owns one
// packed index: it finds that last preimage and evaluates the reference's
// expression for it, product by product and sum by sum in the same order
// (__dmul_rn / __dadd_rn: no contraction), so the result is bit-identical.
#include "v2b_orbital.cuh"

namespace v2b {

__device__ __forceinline__ int64_t tri_idx(int64_t i, int64_t j) {
    return i >= j ? i * (i + 1) / 2 + j : j * (j + 1) / 2 + i;
}

// i >= j with i (i + 1) / 2 + j = t
__device__ __forceinline__ void tri_decode(int64_t t, int &i, int &j) {
    int64_t a = (int64_t)((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
    while (a * (a + 1) / 2 > t) a--;
    while ((a + 1) * (a + 2) / 2 <= t) a++;
    i = (int)a;
    j = (int)(t - a * (a + 1) / 2);
}

__global__ void __launch_bounds__(256)
    pack_spatial_density_kernel(const double *__restrict__ x, PackArgs a, double *__restrict__ d2,
                                double *__restrict__ d1) {
    const int n = a.n;
    const int64_t gab = (int64_t)n * n, gaa = (int64_t)n * (n - 1) / 2;
    const int64_t g00 = (int64_t)n * (n + 1) / 2, nd2 = g00 * (g00 + 1) / 2, nd1 = g00;
    for (int64_t id = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; id < nd2 + nd1;
         id += (int64_t)gridDim.x * blockDim.x) {
        if (id >= nd2) {   // d1: i <= j, INDEX(i, j) (v2rdm_solver.cc:3203-3215)
            int jj, ii;
            tri_decode(id - nd2, jj, ii);   // jj >= ii
            d1[id - nd2] = __dadd_rn(x[a.d1a + (int64_t)ii * n + jj], x[a.d1b + (int64_t)ii * n + jj]);
            continue;
        }
        int P0, R0;
        tri_decode(id, P0, R0);   // packed pair (P0 >= R0) of "00" geminals
        int pa, pb, ra, rb;
        tri_decode(P0, pa, pb);
        tri_decode(R0, ra, rb);
        // preimages: (i, k) from one geminal in either order, (j, l) from the
        // other in either order; keep the one the reference visits last
        int64_t best = -1;
        int bi = 0, bj = 0, bk = 0, bl = 0;
        for (int sw = 0; sw < 2; sw++) {
            const int f0 = sw ? ra : pa, f1 = sw ? rb : pb, s0 = sw ? pa : ra, s1 = sw ? pb : rb;
            for (int o1 = 0; o1 < 2; o1++)
                for (int o2 = 0; o2 < 2; o2++) {
                    const int i = o1 ? f1 : f0, k = o1 ? f0 : f1;
                    const int j = o2 ? s1 : s0, l = o2 ? s0 : s1;
                    // geminal ij holds (first, second) = (ij % n, ij / n)
                    const int64_t L = ((int64_t)j * n + i) * gab + ((int64_t)l * n + k);
                    if (L > best) {
                        best = L;
                        bi = i; bj = j; bk = k; bl = l;
                    }
                }
        }
        const int i = bi, j = bj, k = bk, l = bl;
        auto iab = [&](int p, int q) { return (int64_t)q * n + p; };
        auto iaa = [&](int p, int q) { return (int64_t)a.ibas_aa[p * n + q]; };
        const double dlj = 1.0 - (double)(l == j), dik = 1.0 - (double)(i == k);
        const double *ab = x + a.d2ab;
        auto half = [&](double v) { return __dmul_rn(0.5, v); };
        double val = 0.0;
        val = __dadd_rn(val, half(ab[iab(i, j) * gab + iab(k, l)]));
        val = __dadd_rn(val, __dmul_rn(half(ab[iab(k, j) * gab + iab(i, l)]), dlj));
        val = __dadd_rn(val, __dmul_rn(half(ab[iab(i, l) * gab + iab(k, j)]), dik));
        val = __dadd_rn(val, __dmul_rn(__dmul_rn(half(ab[iab(k, l) * gab + iab(i, j)]), dlj), dik));
        val = __dadd_rn(val, half(ab[iab(j, i) * gab + iab(l, k)]));
        val = __dadd_rn(val, __dmul_rn(half(ab[iab(j, k) * gab + iab(l, i)]), dlj));
        val = __dadd_rn(val, __dmul_rn(half(ab[iab(l, i) * gab + iab(j, k)]), dik));
        val = __dadd_rn(val, __dmul_rn(__dmul_rn(half(ab[iab(l, k) * gab + iab(j, i)]), dlj), dik));
        const double *aa = x + a.d2aa, *bb = x + a.d2bb;
        if (i != j && k != l) {
            // 0.5 * sij * skl * x[...] (* dlj * dik), left to right
            const double c = __dmul_rn(__dmul_rn(0.5, (double)(i < j ? 1 : -1)), (double)(k < l ? 1 : -1));
            const int64_t ij = iaa(i, j), kl = iaa(k, l);
            val = __dadd_rn(val, __dmul_rn(c, aa[ij * gaa + kl]));
            val = __dadd_rn(val, __dmul_rn(__dmul_rn(__dmul_rn(c, aa[kl * gaa + ij]), dlj), dik));
            val = __dadd_rn(val, __dmul_rn(c, bb[ij * gaa + kl]));
            val = __dadd_rn(val, __dmul_rn(__dmul_rn(__dmul_rn(c, bb[kl * gaa + ij]), dlj), dik));
        }
        if (k != j && i != l) {
            const double c = __dmul_rn(__dmul_rn(0.5, (double)(k < j ? 1 : -1)), (double)(i < l ? 1 : -1));
            const int64_t kj = iaa(k, j), il = iaa(i, l);
            val = __dadd_rn(val, __dmul_rn(__dmul_rn(c, aa[kj * gaa + il]), dlj));
            val = __dadd_rn(val, __dmul_rn(__dmul_rn(c, aa[il * gaa + kj]), dik));
            val = __dadd_rn(val, __dmul_rn(__dmul_rn(c, bb[kj * gaa + il]), dlj));
            val = __dadd_rn(val, __dmul_rn(__dmul_rn(c, bb[il * gaa + kj]), dik));
        }
        if (tri_idx(i, k) != tri_idx(j, l)) val = __dmul_rn(val, 2.0);
        d2[id] = val;
    }
}

}  // namespace v2b
