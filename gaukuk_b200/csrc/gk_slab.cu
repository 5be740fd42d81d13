// gk_slab.cu -- device side of a 2D grid split into y-slabs: the halo
// exchange of the two ghost rows per side between slabs, and the CFL maximum
// over slabs that keeps one global dt (sim.cpp:77-81: dt = CFL*drmin/cmax
// with cmax over the whole grid).
//
// A slab is an ordinary fused-2D handle whose y sides between slabs (and
// both y sides under periodic y, which becomes a ring) are filled by the
// exchange instead of the ghost fill, and whose last stage defers its step
// epilogue until the maximum over all slabs is known.  Every ghost value the
// stage kernel reads is then the value the undivided grid would hold, so the
// slabs' results are the single grid's, bit for bit.
#include "gk_internal.h"

namespace gk {

namespace {

__global__ void k_slab_halo(const SlabDev* __restrict__ sd, int role, int ib, int nx, int pitch) {
    const SlabDev& me = sd[blockIdx.z];
    if (!me.tm->active) return;
    const int side = blockIdx.y / 10, rem = blockIdx.y % 10;
    const int v = rem >> 1, r = rem & 1;
    const int nb = side == 0 ? me.lower : me.upper;
    if (nb < 0) return;
    const SlabDev& src = sd[nb];
    const int i = ib + blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ib + nx) return;
    // lower ghosts jb-2, jb-1 <- the lower neighbour's last rows je-2, je-1;
    // upper ghosts je, je+1 <- the upper neighbour's first rows jb, jb+1
    const int dst_row = side == 0 ? me.jb - 2 + r : me.je + r;
    const int src_row = side == 0 ? src.je - 2 + r : src.jb + r;
    me.buf[role][v * me.vstride + (long long)dst_row * pitch + i] =
        src.buf[role][v * src.vstride + (long long)src_row * pitch + i];
}

__global__ void k_slab_reduce(SlabDev* __restrict__ sd, int n, int which) {
    unsigned long long m = 0;
    int st = 0;
    for (int k = 0; k < n; ++k) {
        const DevTime* t = sd[k].tm;
        const unsigned long long b =
            which ? (unsigned long long)__double_as_longlong(t->cmax_last) : t->cmax_acc;
        m = b > m ? b : m;
        st |= t->status;
    }
    for (int k = 0; k < n; ++k) {
        DevTime* t = sd[k].tm;
        if (which) t->cmax_last = __longlong_as_double((long long)m);
        else t->cmax_acc = m;
        t->status |= st;
    }
}

__global__ void k_slab_pack(const double* __restrict__ u, double* __restrict__ lo,
                            double* __restrict__ hi, Geom g, const DevTime* __restrict__ tm) {
    if (!tm->active) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.nx) return;
    const int v = blockIdx.y >> 1, r = blockIdx.y & 1;
    const long long o = (long long)(v * 2 + r) * g.nx + i;
    const double* p = u + v * g.vstride + g.ib + i;
    lo[o] = p[(long long)(g.jb + r) * g.pitch];
    hi[o] = p[(long long)(g.je - 2 + r) * g.pitch];
}

__global__ void k_slab_unpack(double* __restrict__ u, const double* __restrict__ lo,
                              const double* __restrict__ hi, Geom g,
                              const DevTime* __restrict__ tm) {
    if (!tm->active) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.nx) return;
    const int v = blockIdx.y >> 1, r = blockIdx.y & 1;
    const long long o = (long long)(v * 2 + r) * g.nx + i;
    double* p = u + v * g.vstride + g.ib + i;
    if (lo) p[(long long)(g.jb - 2 + r) * g.pitch] = lo[o];
    if (hi) p[(long long)(g.je + r) * g.pitch] = hi[o];
}

__global__ void k_slab_red_pack(const DevTime* __restrict__ tm, unsigned long long* red, int which) {
    red[0] = which ? (unsigned long long)__double_as_longlong(tm->cmax_last) : tm->cmax_acc;
    red[1] = (unsigned long long)(unsigned)tm->status;
}

__global__ void k_slab_red_unpack(DevTime* __restrict__ tm, const unsigned long long* red,
                                  int which) {
    if (which) tm->cmax_last = __longlong_as_double((long long)red[0]);
    else tm->cmax_acc = red[0];
    tm->status |= (int)red[1];
}

}  // namespace

void launch_slab_halo(const SlabDev* sd, int n, int role, const Geom& g, cudaStream_t s) {
    const int threads = 128;
    dim3 grid((g.nx + threads - 1) / threads, 20, n);
    k_slab_halo<<<grid, threads, 0, s>>>(sd, role, g.ib, g.nx, g.pitch);
}

void launch_slab_reduce(const SlabDev* sd, int n, int which, cudaStream_t s) {
    k_slab_reduce<<<1, 1, 0, s>>>(const_cast<SlabDev*>(sd), n, which);
}

void launch_slab_pack(const double* u, double* send_lo, double* send_hi, const Geom& g,
                      const DevTime* tm, cudaStream_t s) {
    const int threads = 128;
    k_slab_pack<<<dim3((g.nx + threads - 1) / threads, 10), threads, 0, s>>>(u, send_lo, send_hi,
                                                                             g, tm);
}

void launch_slab_unpack(double* u, const double* recv_lo, const double* recv_hi, const Geom& g,
                        const DevTime* tm, cudaStream_t s) {
    const int threads = 128;
    k_slab_unpack<<<dim3((g.nx + threads - 1) / threads, 10), threads, 0, s>>>(u, recv_lo,
                                                                               recv_hi, g, tm);
}

void launch_slab_red_pack(const DevTime* tm, unsigned long long* red, int which, cudaStream_t s) {
    k_slab_red_pack<<<1, 1, 0, s>>>(tm, red, which);
}

void launch_slab_red_unpack(DevTime* tm, const unsigned long long* red, int which,
                            cudaStream_t s) {
    k_slab_red_unpack<<<1, 1, 0, s>>>(tm, red, which);
}

}  // namespace gk
