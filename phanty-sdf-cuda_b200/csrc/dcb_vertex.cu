// dcb_vertex.cu — the FP32 cyclic-Jacobi solve of the cells whose normal equations the band
// kernel (dcb_band.cu) could not certify as rank 1.
//
// Semantics: Cell::update / solve_quadratic_system (src/cpp/Cell.cpp:284-361): the truncated
// pseudo-inverse of A^T A (singular values <= svd_threshold dropped) about the centroid. A cell
// whose retained spectrum is ill-conditioned, or has an eigenvalue within a relative band of
// the threshold (the rank decision is ambiguous in FP32), is listed for the FP64 path
// (dcb_vertex64.cu), which repeats the CPU arithmetic.
#include "dcb_qef.cuh"

namespace dcb {

// ---- k_cell_jacobi ----------------------------------------------------------------------

// Cyclic Jacobi eigen-decomposition of a symmetric 3x3 (Golub & Van Loan 8.5) in FP32.
__device__ __forceinline__ void jacobi3f(float a[3][3], float V[3][3]) {
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) V[r][c] = (r == c) ? 1.f : 0.f;
    for (int sweep = 0; sweep < 8; ++sweep) {
        const float off = a[0][1] * a[0][1] + a[0][2] * a[0][2] + a[1][2] * a[1][2];
        const float diag = a[0][0] * a[0][0] + a[1][1] * a[1][1] + a[2][2] * a[2][2];
        if (off <= 1e-14f * diag || off == 0.f) break;
#pragma unroll
        for (int pq = 0; pq < 3; ++pq) {
            const int p = pq == 2 ? 1 : 0;
            const int q = pq == 0 ? 1 : 2;
            const float apq = a[p][q];
            if (apq == 0.f) continue;
            const float theta = (a[q][q] - a[p][p]) / (2.f * apq);
            const float t = (theta >= 0.f ? 1.f : -1.f) / (fabsf(theta) + sqrtf(theta * theta + 1.f));
            const float c = rsqrtf(t * t + 1.f), s = t * c;
#pragma unroll
            for (int r = 0; r < 3; ++r) {
                const float arp = a[r][p], arq = a[r][q];
                a[r][p] = c * arp - s * arq;
                a[r][q] = s * arp + c * arq;
            }
#pragma unroll
            for (int r = 0; r < 3; ++r) {
                const float apr = a[p][r], aqr = a[q][r];
                a[p][r] = c * apr - s * aqr;
                a[q][r] = s * apr + c * aqr;
            }
#pragma unroll
            for (int r = 0; r < 3; ++r) {
                const float vrp = V[r][p], vrq = V[r][q];
                V[r][p] = c * vrp - s * vrq;
                V[r][q] = s * vrp + c * vrq;
            }
        }
    }
}

__global__ void __launch_bounds__(128)
k_cell_jacobi(QefParams P) {
    __shared__ unsigned int s_hist[4];
    if (threadIdx.x < 4) s_hist[threadIdx.x] = 0;
    __syncthreads();
    const unsigned int n = *P.hard_count;
    for (unsigned int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const uint32_t r = P.hard_list[t];
        const float4 d0 = P.hard_data[3 * (size_t)t], d1 = P.hard_data[3 * (size_t)t + 1], d2 = P.hard_data[3 * (size_t)t + 2];
        int i, j, k;
        unpack_cell(P.list[r], i, j, k);
        float A[3][3] = {{d0.x, d0.y, d0.z}, {d0.y, d0.w, d1.x}, {d0.z, d1.x, d1.y}};
        const float R0 = d1.z, R1 = d1.w, R2 = d2.x;
        float EV[3][3];
        jacobi3f(A, EV);
        const float lam[3] = {fabsf(A[0][0]), fabsf(A[1][1]), fabsf(A[2][2])};
        int rank = 0;
        bool near = false;
        float lmax = 0.f, lmin_ret = 3.4e38f, wx = 0.f, wy = 0.f, wz = 0.f;
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            lmax = fmaxf(lmax, lam[q]);
            near |= fabsf(lam[q] - P.thr) <= P.band * P.thr;
            if (lam[q] > P.thr) {
                ++rank;
                lmin_ret = fminf(lmin_ret, lam[q]);
                const float proj = (EV[0][q] * R0 + EV[1][q] * R1 + EV[2][q] * R2) / lam[q];
                wx += EV[0][q] * proj; wy += EV[1][q] * proj; wz += EV[2][q] * proj;
            }
        }
        const bool ill_cond = rank >= 1 && lmax > P.cond_max * lmin_ret;
        atomicAdd(&s_hist[rank], 1u);
        if (near || ill_cond) {
            const unsigned int slot = atomicAdd(P.esc_count, 1u);
            P.esc_list[slot] = r;
        }
        const GridDesc g = P.B.slots[slot_of_rank(P.B, r)].g;
        const float wx1 = width_axis(g, 0, i), wy1 = width_axis(g, 1, j), wz1 = width_axis(g, 2, k);
        store_vertex(P.V, g, r, i, j, k, d2.y + wx, d2.z + wy * (wx1 / wy1), d2.w + wz * (wx1 / wz1));
        P.vclass[r] = kVcJacobi;
    }
    __syncthreads();
    if (threadIdx.x < 4 && s_hist[threadIdx.x]) atomicAdd(P.rank_hist + threadIdx.x, (unsigned long long)s_hist[threadIdx.x]);
}

cudaError_t launch_cell_jacobi(const QefParams& P, long long max_items, int num_sms, cudaStream_t s) {
    if (max_items <= 0) return cudaSuccess;
    long long blocks = (max_items + 127) / 128;
    const long long cap = (long long)num_sms * 16;
    if (blocks > cap) blocks = cap;
    k_cell_jacobi<<<(unsigned)blocks, 128, 0, s>>>(P);
    return cudaGetLastError();
}

}  // namespace dcb
