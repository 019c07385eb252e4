// Exhaustive check of the backprojectors' reciprocal (rcp_rn_nr in
// jenhine_b200/csrc/bp_common.cuh) against CUDA's correctly rounded
// __frcp_rn: every float w whose reciprocal is a normal float, both signs
// (exponent fields 1..252, 4.23e9 values).  Prints the count of mismatches and
// the first few; exit status 0 when there are none.  Built and run by
// tests/test_reciprocal.py.
#include <cstdio>
#include <cstring>

#include "bp_common.cuh"

__global__ void check(unsigned n, unsigned long long* bad, unsigned* firsts) {
    for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const unsigned bits = (1u << 23) + i;
        for (unsigned sgn = 0; sgn < 2; ++sgn) {
            const float w = __uint_as_float(bits | (sgn << 31));
            if (__float_as_uint(__frcp_rn(w)) != __float_as_uint(jfdk::rcp_rn_nr(w))) {
                const unsigned long long k = atomicAdd(bad, 1ull);
                if (k < 8) firsts[k] = bits | (sgn << 31);
            }
        }
    }
}

int main() {
    const unsigned n = 252u << 23;   // i + stride stays below 2^32
    unsigned long long* bad = nullptr;
    unsigned* firsts = nullptr;
    if (cudaMalloc(&bad, sizeof(*bad)) != cudaSuccess || cudaMalloc(&firsts, 8 * sizeof(*firsts)) != cudaSuccess) {
        std::printf("allocation failed\n");
        return 2;
    }
    cudaMemset(bad, 0, sizeof(*bad));
    cudaMemset(firsts, 0, 8 * sizeof(*firsts));
    check<<<148 * 8, 256>>>(n, bad, firsts);
    const cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        std::printf("CUDA error: %s\n", cudaGetErrorString(e));
        return 2;
    }
    unsigned long long hb = 0;
    unsigned hf[8] = {0};
    cudaMemcpy(&hb, bad, sizeof(hb), cudaMemcpyDeviceToHost);
    cudaMemcpy(hf, firsts, sizeof(hf), cudaMemcpyDeviceToHost);
    std::printf("checked %llu values, mismatches %llu\n", 2ull * n, hb);
    for (int k = 0; k < 8 && (unsigned long long)k < hb; ++k) {
        float f;
        std::memcpy(&f, &hf[k], 4);
        std::printf("  w = %.9g (bits %08x)\n", f, hf[k]);
    }
    cudaFree(bad);
    cudaFree(firsts);
    return hb ? 1 : 0;
}
