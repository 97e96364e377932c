// A C++ caller of the TAL-SH C API, written the way the reference's own
// test_talsh_c (test.cpp:38-165) uses it: Host tensors constructed with values,
// an asynchronous contraction on GPU 0 with COPY_MTT polled with
// talshTaskComplete, the result moved back with talshTensorPlace, and the
// 1-norm checked against its analytic value.  It compiles against
// include/talsh.h unchanged and links libtalsh.so.
#include <cmath>
#include <cstdio>

#include "talsh.h"

int main() {
  const int V = 40, O = 20;
  size_t host_buffer_size = 1 << 24;
  int host_arg_max = 0, ngpu = 0;
  if (talshDeviceCount(DEV_NVIDIA_GPU, &ngpu) != TALSH_SUCCESS || ngpu < 1) { std::printf("FAIL no gpu\n"); return 1; }
  int gpu_list[1] = {0};
  if (talshInit(&host_buffer_size, &host_arg_max, 1, gpu_list, 0, NULL, 0, NULL) != TALSH_SUCCESS) return 2;
  const int dims0[] = {V, V, O, O}, dims1[] = {V, V, V, V}, dims2[] = {O, V, O, V};
  talsh_tens_t t0, t1, t2;
  talshTensorClean(&t0); talshTensorClean(&t1); talshTensorClean(&t2);
  if (talshTensorConstruct(&t0, R8, 4, dims0, talshFlatDevId(DEV_HOST, 0), NULL, -1, NULL, 0.0)) return 3;
  if (talshTensorConstruct(&t1, R8, 4, dims1, talshFlatDevId(DEV_HOST, 0), NULL, -1, NULL, 0.001)) return 4;
  if (talshTensorConstruct(&t2, R8, 4, dims2, talshFlatDevId(DEV_HOST, 0), NULL, -1, NULL, 0.01)) return 5;
  const double gflops = std::sqrt((double)talshTensorVolume(&t0) * (double)talshTensorVolume(&t1) *
                                  (double)talshTensorVolume(&t2)) * 2.0 / 1e9;
  const double theor_norm1 = gflops * 0.01 * 0.001 * 1e9;
  talsh_task_t task;
  talshTaskClean(&task);
  int errc = talshTensorContract("D(a,b,i,j)+=L(c,b,d,a)*R(j,d,i,c)", &t0, &t1, &t2, 2.0, 0.0, 0, DEV_NVIDIA_GPU,
                                 COPY_MTT, YEP, &task);
  if (errc) { std::printf("FAIL schedule %d\n", errc); return 6; }
  int sts = 0, done = NOPE;
  while (done != YEP && errc == TALSH_SUCCESS) done = talshTaskComplete(&task, &sts, &errc);
  if (errc != TALSH_SUCCESS || sts != TALSH_TASK_COMPLETED) { std::printf("FAIL task %d %d\n", errc, sts); return 7; }
  double total = 0.0;
  if (talshTaskTime(&task, &total)) return 8;
  talshTaskDestruct(&task);
  if (talshTensorPlace(&t0, 0, DEV_HOST, NULL, COPY_M)) return 9;
  const double norm1 = talshTensorImageNorm1_cpu(&t0);
  std::printf("norm1 %.15e theory %.15e time %.6f s GFlop/s %.1f\n", norm1, theor_norm1, total, gflops / total);
  const bool ok = std::fabs(norm1 - theor_norm1) <= 1e-10 * theor_norm1;
  talshTensorDestruct(&t2); talshTensorDestruct(&t1); talshTensorDestruct(&t0);
  if (talshShutdown()) return 10;
  std::printf(ok ? "PASS\n" : "FAIL norm\n");
  return ok ? 0 : 11;
}
