// bench_int_pipes.cu -- integer-pipe throughput of the GPU (warp-instructions per SM-cycle) for LOP3, IMAD,
// SHF, PRMT, IADD, a LOP3+IMAD mix, shared-memory loads and shuffles.  bench.py uses the LOP3 rate
// as the peak of its integer-ALU roofline (`python bench.py --int-peak` builds and runs this file).
// Every access is in bounds by construction: one output word per thread, a 4 KB shared buffer
// indexed with & 255.
#include <cstdio>
#include <cstdint>
#include <cuda_runtime.h>

#define CHAINS 8
#define UNROLL 16

template <int KIND>
__global__ void kern(uint32_t *out, uint32_t seed, int iters, long long *cyc) {
    __shared__ uint4 sm[256];
    for (int i = threadIdx.x; i < 256; i += blockDim.x) sm[i] = make_uint4(i * seed, i + seed, i ^ seed, i * 7);
    __syncthreads();
    uint32_t a[CHAINS];
#pragma unroll
    for (int c = 0; c < CHAINS; c++) a[c] = seed * (threadIdx.x + 17 * c + 1);
    uint32_t b = seed * 3 + threadIdx.x, d = seed * 5 + blockIdx.x;
    long long t0 = clock64();
    for (int it = 0; it < iters; it++) {
#pragma unroll
        for (int u = 0; u < UNROLL; u++) {
#pragma unroll
            for (int c = 0; c < CHAINS; c++) {
                if (KIND == 0) asm volatile("lop3.b32 %0, %0, %1, %2, 0x96;" : "+r"(a[c]) : "r"(b), "r"(d));
                if (KIND == 1) asm volatile("mad.lo.u32 %0, %0, %1, %2;" : "+r"(a[c]) : "r"(b), "r"(d));
                if (KIND == 2) asm volatile("shf.l.wrap.b32 %0, %0, %1, %2;" : "+r"(a[c]) : "r"(b), "r"(d));
                if (KIND == 3) asm volatile("prmt.b32 %0, %0, %1, %2;" : "+r"(a[c]) : "r"(b), "r"(d));
                if (KIND == 4) asm volatile("add.u32 %0, %0, %1;\n\tadd.u32 %0, %0, %2;" : "+r"(a[c]) : "r"(b), "r"(d));
                if (KIND == 5) {  // LOP3 and IMAD interleaved on alternate chains
                    if (c & 1) asm volatile("mad.lo.u32 %0, %0, %1, %2;" : "+r"(a[c]) : "r"(b), "r"(d));
                    else asm volatile("lop3.b32 %0, %0, %1, %2, 0x96;" : "+r"(a[c]) : "r"(b), "r"(d));
                }
                if (KIND == 6) {  // LDS.128, per-lane distinct 16B chunk (conflict-free), then a LOP3 use
                    uint4 v = sm[(threadIdx.x + 8 * c + u + it) & 255];  // independent of the chain
                    a[c] ^= v.x ^ v.w;
                }
                if (KIND == 7) a[c] = __shfl_xor_sync(0xffffffffu, a[c], 1 + (c & 15)) + 1;
                if (KIND == 8) {  // LDS.128 broadcast (same address in the warp)
                    uint4 v = sm[(a[0] >> 24) & 255];
                    a[c] ^= v.y;
                }
            }
        }
    }
    long long t1 = clock64();
    uint32_t x = 0;
#pragma unroll
    for (int c = 0; c < CHAINS; c++) x ^= a[c];
    out[blockIdx.x * blockDim.x + threadIdx.x] = x;
    if (threadIdx.x == 0) cyc[blockIdx.x] = t1 - t0;
}

template <int KIND>
void run(const char *name, int nsm, double instr_per_inner) {
    int threads = 256, blocks = nsm * 8, iters = 2000;
    uint32_t *out;
    long long *cyc;
    cudaMalloc(&out, sizeof(uint32_t) * threads * blocks);
    cudaMalloc(&cyc, sizeof(long long) * blocks);
    kern<KIND><<<blocks, threads>>>(out, 12345u, 10, cyc);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0);
    kern<KIND><<<blocks, threads>>>(out, 12345u, iters, cyc);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms;
    cudaEventElapsedTime(&ms, e0, e1);
    long long *hc = new long long[blocks];
    cudaMemcpy(hc, cyc, sizeof(long long) * blocks, cudaMemcpyDeviceToHost);
    long long mx = 0;
    for (int i = 0; i < blocks; i++) mx = hc[i] > mx ? hc[i] : mx;
    double warp_instr = (double)blocks * (threads / 32) * iters * UNROLL * CHAINS * instr_per_inner;
    double per_sm_cycle = warp_instr / nsm / (double)mx;
    double mhz = (double)mx / (ms * 1e3);
    printf("%-22s %8.3f ms  %7.3f warp-instr/SM/clk (%6.1f lane-ops/SM/clk)  clk~%.0f MHz  err=%d\n", name, ms,
           per_sm_cycle, per_sm_cycle * 32, mhz, (int)cudaGetLastError());
    delete[] hc;
    cudaFree(out);
    cudaFree(cyc);
}

int main() {
    int dev = 0, nsm = 0;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    printf("SMs: %d\n", nsm);
    run<0>("LOP3", nsm, 1);
    run<1>("IMAD", nsm, 1);
    run<2>("SHF", nsm, 1);
    run<3>("PRMT", nsm, 1);
    run<4>("IADD(x2)", nsm, 2);
    run<5>("LOP3+IMAD 1:1", nsm, 1);
    run<6>("LDS.128+2LOP", nsm, 1);
    run<7>("SHFL+IADD", nsm, 1);
    run<8>("LDS.128 bcast+LOP", nsm, 1);
    return 0;
}
