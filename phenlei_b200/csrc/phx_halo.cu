// Halo exchange of a partitioned grid: rows of the cells one zone sends,
// gathered into a contiguous device buffer, and the same rows scattered into
// the interface ghosts of the zone that receives them.  The reference moves
// the same interface data between zones with Controller::CommunicationInterfaceData
// (CFD/Solver/src/Controller.cpp:3389) and CommunicationDQ (:2874); what it
// sends at each point is listed with the PHX_HALO_* codes in include/phx.h.
//
// Rows are copied bit for bit, so the receiving zone sees exactly the values
// the sending zone holds (FP64 master state, working-precision records).
#include <cuda_runtime.h>
#include <stdint.h>

#include "phx_device.cuh"
#include "phx_internal.h"

namespace phx {

// Row layouts (T = working precision):
//  Q         5 doubles: rho u v w p of the FP64 master state
//  GRADIENT  kG T: the gradient record, slot 15 (padding) carrying the limiter
//  DQ        kD T: the forward-sweep dq record
//  TURB      2 doubles: master nu~, eddy viscosity
template <class T>
size_t halo_row_bytes(int field)
{
    switch (field) {
    case PHX_HALO_Q: return 5 * sizeof(double);
    case PHX_HALO_GRADIENT: return kG * sizeof(T);
    case PHX_HALO_DQ: return kD * sizeof(T);
    case PHX_HALO_TURB: return 2 * sizeof(double);
    default: return 0;
    }
}

template <class T>
__global__ void __launch_bounds__(kThreads) halo_pack_kernel(DevGrid g, int field, const double *q64, Work<T> w,
                                                             TurbWork<T> t, const int *send, int n,
                                                             unsigned char *buf)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int c = send[i];
    const int nt = g.nTotal;
    if (field == PHX_HALO_Q) {
        double *o = reinterpret_cast<double *>(buf) + (size_t)i * 5;
#pragma unroll
        for (int k = 0; k < 5; ++k) o[k] = q64[(size_t)k * nt + c];
    } else if (field == PHX_HALO_GRADIENT) {
        T *o = reinterpret_cast<T *>(buf) + (size_t)i * kG;
        const T *gr = w.grec + (size_t)c * kG;
#pragma unroll
        for (int k = 0; k < kG; ++k) o[k] = gr[k];
        o[15] = w.qrec[(size_t)c * kQ + 7];
    } else if (field == PHX_HALO_DQ) {
        T *o = reinterpret_cast<T *>(buf) + (size_t)i * kD;
        const T *d = w.dqfwd + (size_t)c * kD;
#pragma unroll
        for (int k = 0; k < kD; ++k) o[k] = d[k];
    } else if (field == PHX_HALO_TURB) {
        double *o = reinterpret_cast<double *>(buf) + (size_t)i * 2;
        o[0] = t.qt64[c];
        o[1] = (double)w.trec[(size_t)c * kTr + 1];
    }
}

template <class T>
__global__ void __launch_bounds__(kThreads) halo_unpack_kernel(DevGrid g, NsConst cst, int field, double *q64,
                                                               Work<T> w, TurbWork<T> t, const int *recv, int n,
                                                               const unsigned char *buf)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int c = recv[i];
    const int nt = g.nTotal;
    if (field == PHX_HALO_Q) {
        // the ghost's FP64 state and its working record (state, c2, hm); the
        // limiter slot keeps the last GRADIENT exchange's value
        const double *v = reinterpret_cast<const double *>(buf) + (size_t)i * 5;
        T s[5];
#pragma unroll
        for (int k = 0; k < 5; ++k) {
            q64[(size_t)k * nt + c] = v[k];
            s[k] = (T)v[k];
        }
        put_state<T>(w.qrec + (size_t)c * kQ, s, (T)cst.gama);
    } else if (field == PHX_HALO_GRADIENT) {
        const T *v = reinterpret_cast<const T *>(buf) + (size_t)i * kG;
        T *gr = w.grec + (size_t)c * kG;
#pragma unroll
        for (int k = 0; k < kG; ++k) gr[k] = k == 15 ? T(0) : v[k];
        w.qrec[(size_t)c * kQ + 7] = v[15];
    } else if (field == PHX_HALO_DQ) {
        const T *v = reinterpret_cast<const T *>(buf) + (size_t)i * kD;
        T *d = w.dqfwd + (size_t)c * kD;
#pragma unroll
        for (int k = 0; k < kD; ++k) d[k] = v[k];
    } else if (field == PHX_HALO_TURB) {
        const double *v = reinterpret_cast<const double *>(buf) + (size_t)i * 2;
        t.qt64[c] = v[0];
        w.trec[(size_t)c * kTr] = (T)v[0];
        w.trec[(size_t)c * kTr + 1] = (T)v[1];
    }
}

template <class T>
void launch_halo_pack(const DevGrid &g, int field, const double *q64, const Work<T> &w, const TurbWork<T> &t,
                      const int *send, int n, unsigned char *buf, cudaStream_t s)
{
    if (n <= 0) return;
    halo_pack_kernel<T><<<(n + kThreads - 1) / kThreads, kThreads, 0, s>>>(g, field, q64, w, t, send, n, buf);
}

template <class T>
void launch_halo_unpack(const DevGrid &g, const NsConst &c, int field, double *q64, const Work<T> &w,
                        const TurbWork<T> &t, const int *recv, int n, const unsigned char *buf, cudaStream_t s)
{
    if (n <= 0) return;
    halo_unpack_kernel<T><<<(n + kThreads - 1) / kThreads, kThreads, 0, s>>>(g, c, field, q64, w, t, recv, n, buf);
}

#define PHX_HALO_INSTANTIATE(T)                                                                                  \
    template size_t halo_row_bytes<T>(int);                                                                      \
    template void launch_halo_pack<T>(const DevGrid &, int, const double *, const Work<T> &, const TurbWork<T> &, \
                                      const int *, int, unsigned char *, cudaStream_t);                          \
    template void launch_halo_unpack<T>(const DevGrid &, const NsConst &, int, double *, const Work<T> &,        \
                                        const TurbWork<T> &, const int *, int, const unsigned char *, cudaStream_t);
PHX_HALO_INSTANTIATE(float)
PHX_HALO_INSTANTIATE(double)

}  // namespace phx
