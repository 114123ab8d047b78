// Built and run by test_gpu_sincos.py: for every float x in [0, 6.2832f]
// (every angle, in radians, that the S3 orientation step can produce),
// counts the inputs where sincos((double)x) differs from (sin, cos) of
// (double)x, bit for bit as doubles. Prints "mismatch <count>".
#include <cstdio>
#include <cstring>

__global__ void count_mismatch(unsigned n, unsigned long long* bad) {
    unsigned long long local = 0;
    for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double x = static_cast<double>(__uint_as_float(i));
        double s, c;
        sincos(x, &s, &c);
        local += __double_as_longlong(c) != __double_as_longlong(cos(x)) ||
                 __double_as_longlong(s) != __double_as_longlong(sin(x));
    }
    atomicAdd(bad, local);
}

int main() {
    const float top = 6.2832f;
    unsigned n;
    std::memcpy(&n, &top, sizeof(n));
    n += 1;  // bit patterns 0 .. top, all nonnegative floats up to top
    unsigned long long* bad = nullptr;
    unsigned long long host = ~0ull;
    if (cudaMalloc(&bad, sizeof(host)) != cudaSuccess || cudaMemset(bad, 0, sizeof(host)) != cudaSuccess) return 1;
    count_mismatch<<<148 * 8, 256>>>(n, bad);
    if (cudaMemcpy(&host, bad, sizeof(host), cudaMemcpyDeviceToHost) != cudaSuccess) return 1;
    std::printf("inputs %u mismatch %llu\n", n, host);
    cudaFree(bad);
    return 0;
}
