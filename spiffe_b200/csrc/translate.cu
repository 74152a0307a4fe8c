// spiffe_b200/csrc/translate.cu -- the moving window (translate_problem,
// translate.c:40-197) on the device.
//
// After each push the reference looks for any particle past z_trigger
// (translate.c:51-57); if there is one, the problem moves by one dz: every
// field row of the TM (and TE) set moves down one row, the top row becomes
// zero, and zmin, zmax and the trigger grow by dz (:123-196).  Metal flags,
// imposed fields, Psi and Q stay where they are.  Here one kernel raises a
// flag when a particle is past the trigger, the host reads it, and the shift
// is two device copies per array through a scratch buffer.  The split form
// stores positions as a cell index relative to zmin, so its particles' cells
// move down one row too, as do the current rows it has already deposited for
// the next step.
#include "modules.cuh"
#include "split32.cuh"

namespace {

constexpr int T = 256;

__global__ void __launch_bounds__(T) k_beyond64(const double *__restrict__ z, const DevCounts *cnt, double trigger,
                                                int *flag)
{
  const long long np = cnt->np;
  for (long long ip = (long long)blockIdx.x * T + threadIdx.x; ip < np; ip += (long long)gridDim.x * T)
    if (z[ip] > trigger) {
      *flag = 1;
      return;
    }
}

__global__ void __launch_bounds__(T) k_beyond32(const int32_t *__restrict__ cell, const float *__restrict__ fz,
                                                const DevCounts *cnt, double zmin, double dz, double trigger,
                                                int *flag)
{
  const long long np = cnt->np;
  for (long long ip = (long long)blockIdx.x * T + threadIdx.x; ip < np; ip += (long long)gridDim.x * T)
    if (zmin + ((double)s32_iz(cell[ip]) + fz[ip]) * dz > trigger) {
      *flag = 1;
      return;
    }
}

__global__ void __launch_bounds__(T) k_cells_down32(int32_t *cell, const DevCounts *cnt)
{
  const long long np = cnt->np;
  for (long long ip = (long long)blockIdx.x * T + threadIdx.x; ip < np; ip += (long long)gridDim.x * T)
    cell[ip] = s32_cell(s32_iz(cell[ip]) - 1, s32_ir(cell[ip]));
}

// the deposited rows [lo, hi] move down one; row 0's current leaves the mesh
__global__ void k_jbox_down(int *jbox)
{
  int lo = jbox[0], hi = jbox[1];
  if (lo > hi)
    return;
  lo = lo > 0 ? lo - 1 : 0;
  hi -= 1;
  if (hi < lo) {
    lo = 0x7fffffff;
    hi = -1;
  }
  jbox[0] = lo;
  jbox[1] = hi;
}

unsigned grid_for(long long np_bound)
{
  const long long b = (np_bound + T - 1) / T;
  return (unsigned)(b < 1 ? 1 : (b > 148 * 8 ? 148 * 8 : b));
}

} // namespace

extern "C" int spiffe_beyond64(const double *z, const DevCounts *cnt, long long np_bound, double trigger, int *flag,
                               cudaStream_t s)
{
  k_beyond64<<<grid_for(np_bound), T, 0, s>>>(z, cnt, trigger, flag);
  spiffe_note_launches(1);
  return (int)cudaGetLastError();
}

extern "C" int s32_beyond(const int32_t *cell, const float *fz, const DevCounts *cnt, long long np_bound, double zmin,
                          double dz, double trigger, int *flag, cudaStream_t s)
{
  k_beyond32<<<grid_for(np_bound), T, 0, s>>>(cell, fz, cnt, zmin, dz, trigger, flag);
  spiffe_note_launches(1);
  return (int)cudaGetLastError();
}

extern "C" int s32_cells_down(int32_t *cell, int *jbox, const DevCounts *cnt, long long np_bound, cudaStream_t s)
{
  k_cells_down32<<<grid_for(np_bound), T, 0, s>>>(cell, cnt);
  spiffe_note_launches(1);
  k_jbox_down<<<1, 1, 0, s>>>(jbox);
  spiffe_note_launches(1);
  return (int)cudaGetLastError();
}

// rows 0..nz of `a` (rows of `row` bytes) move down one row, the last is zeroed
extern "C" int spiffe_rows_down(void *a, size_t row, int nz, void *scratch, cudaStream_t s)
{
  if (!a)
    return 0;
  char *p = (char *)a;
  const size_t n = row * (size_t)nz;
  cudaError_t e = cudaMemcpyAsync(scratch, p + row, n, cudaMemcpyDeviceToDevice, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(p, scratch, n, cudaMemcpyDeviceToDevice, s);
  if (e == cudaSuccess)
    e = cudaMemsetAsync(p + n, 0, row, s);
  return (int)e;
}
