// Checks the assumed f64 mma.sync fragment layouts against an exact CPU product.
#include <cstdio>
#include <cuda_runtime.h>
template <int K> __global__ void probe(const double* A, const double* B, double* D) {
  int lane = threadIdx.x, g = lane >> 2, t = lane & 3;
  constexpr int NQ = K / 4;
  double a[2 * NQ], b[NQ], d[4] = {0, 0, 0, 0};
  for (int q = 0; q < NQ; ++q) for (int h = 0; h < 2; ++h) a[2*q+h] = A[(g + 8*h) * K + t + 4*q];
  for (int q = 0; q < NQ; ++q) b[q] = B[(t + 4*q) * 8 + g];
  if (K == 4)
    asm volatile("mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};"
      : "+d"(d[0]),"+d"(d[1]),"+d"(d[2]),"+d"(d[3]) : "d"(a[0]),"d"(a[1]),"d"(b[0]));
  if (K == 8)
    asm volatile("mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
      : "+d"(d[0]),"+d"(d[1]),"+d"(d[2]),"+d"(d[3]) : "d"(a[0]),"d"(a[1]),"d"(a[2]),"d"(a[3]),"d"(b[0]),"d"(b[1]));
  if (K == 16)
    asm volatile("mma.sync.aligned.m16n8k16.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7,%8,%9,%10,%11}, {%12,%13,%14,%15}, {%0,%1,%2,%3};"
      : "+d"(d[0]),"+d"(d[1]),"+d"(d[2]),"+d"(d[3]) : "d"(a[0]),"d"(a[1]),"d"(a[2]),"d"(a[3]),"d"(a[4]),"d"(a[5]),"d"(a[6]),"d"(a[7]),"d"(b[0]),"d"(b[1]),"d"(b[2]),"d"(b[3]));
  for (int r = 0; r < 4; ++r) D[(g + 8 * (r >> 1)) * 8 + 2 * t + (r & 1)] = d[r];
}
template <int K> int run() {
  double hA[16 * K], hB[K * 8], hD[128], ref[128];
  for (int m = 0; m < 16; ++m) for (int k = 0; k < K; ++k) hA[m * K + k] = m * 37 + k * 3 + 1;
  for (int k = 0; k < K; ++k) for (int n = 0; n < 8; ++n) hB[k * 8 + n] = k * 11 + n * 5 + 2;
  for (int m = 0; m < 16; ++m) for (int n = 0; n < 8; ++n) { double s = 0; for (int k = 0; k < K; ++k) s += hA[m*K+k]*hB[k*8+n]; ref[m*8+n] = s; }
  double *dA, *dB, *dD;
  cudaMalloc(&dA, sizeof hA); cudaMalloc(&dB, sizeof hB); cudaMalloc(&dD, sizeof hD);
  cudaMemcpy(dA, hA, sizeof hA, cudaMemcpyHostToDevice); cudaMemcpy(dB, hB, sizeof hB, cudaMemcpyHostToDevice);
  cudaMemset(dD, 0, sizeof hD);
  probe<K><<<1, 32>>>(dA, dB, dD);
  cudaError_t e = cudaDeviceSynchronize();
  cudaMemcpy(hD, dD, sizeof hD, cudaMemcpyDeviceToHost);
  int bad = 0; for (int i = 0; i < 128; ++i) bad += hD[i] != ref[i];
  printf("m16n8k%d: %s (%d mismatches) err=%s\n", K, bad ? "LAYOUT MISMATCH" : "layout ok", bad, cudaGetErrorString(e));
  cudaFree(dA); cudaFree(dB); cudaFree(dD);
  return bad;
}
int main() { int b = run<4>() + run<8>() + run<16>(); return b ? 1 : 0; }
