// Host side of the phx library: context creation (grid metrics in FP64, the
// cell-to-face lists, the LU-SGS level schedules, boundary classification),
// device memory, and the C ABI declared in include/phx.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>

#include "phx_internal.h"
#include "phx_mlp.h"

namespace phx {
int mlp_loss_grad(const float *params, const float *x, const float *y, int B, float *grad, double &lossOut,
                  cudaStream_t s);
int mlp_param_count();
int mlp_train(const float *X, const float *Y, long long n, int epochs, int batch, float lr, unsigned long long seed,
              MlpHostWeights &wts, float *mean, float *rstd, float *lo, float *hi, float *occ, float &tscale,
              double &lastLoss, cudaStream_t s);
void mlp_pack(const MlpHostWeights &w, std::vector<uint16_t> &w1c, std::vector<uint16_t> &w2c,
              std::vector<uint16_t> &w3c);
}  // namespace phx

using namespace phx;

// Flat model blob of phx_mlp_get / phx_mlp_set: weights (w1 b1 w2 b2 w3 b3 w4
// b4, row-major [out][in]), then mean, 1/std, hull lo, hull hi (6 each), target
// scale, and the hull's occupied (ln chi, ln s) bins (kMlpGrid x kMlpGrid, 0 / 1).
static constexpr int kMlpWeightFloats = sizeof(MlpHostWeights) / sizeof(float);
static constexpr int kMlpBlobFloats = kMlpWeightFloats + 4 * kMlpIn + 1 + kMlpGrid * kMlpGrid;

struct phx_ctx {
    int device = 0;
    int numSMs = 148;
    cudaStream_t stream = nullptr;
    // second stream of the fused driver: the next step's NS boundary and
    // gradient run on it while the SA sweep runs (phx_ns_relaxation)
    cudaStream_t aux = nullptr;
    cudaEvent_t evFork = nullptr, evHead = nullptr;
    std::string err;
    int64_t launches = 0;
    phx_params prm{};
    NsConst nc{};
    int nNode = 0, nFace = 0, nCell = 0, nBFace = 0, nTotal = 0;
    bool mixed = false;
    // geometry in the reference's order (answers phx_get_geometry, derives dt)
    std::vector<double> geom[12];  // xfn yfn zfn area xfc yfc zfc xcc ycc zcc vol skew
    std::vector<void *> allocs;
    DevGrid g{};
    double *q64[2] = {nullptr, nullptr};  // FP64 master state [5][nTotal], storage order
    int cur = 0;
    Work<double> w64{};
    Work<float> w32{};
    TurbWork<double> t64{};
    TurbWork<float> t32{};
    bool sa = false;
    // learned SA source
    bool mlpReady = false;
    MlpDev mlp{};
    std::vector<float> mlpBlob;
    uint16_t *mlpW = nullptr;               // w1c | w2c | w3c (FP16 words)
    float *mlpF = nullptr;                  // b1 | b2 | b3 | w4
    uint8_t *mlpOcc = nullptr;              // occupied hull bins
    unsigned long long *nmlp = nullptr;     // cells that used the learned source (running count)
    double *forces = nullptr;               // [16] wall force sums
    Reduce *red = nullptr;
    int *neglist = nullptr;
    double *tmp = nullptr;                // [5][nTotal] staging buffer in the reference's order
    double *hist = nullptr;
    int histCap = 0;
    bool nodePrev = false;                // GG-node: node values of a previous state are in nrec (slot 5)
    bool turbNodeValid = false;           // GG-node with SA: qtnode holds node values for the next SA gradient
    int step = 0;
    bool haveResidual = false;
    std::vector<int> rankOf;              // storage index of each reference cell
    // partitioned grids (interface faces): the topology and storage maps that
    // phx_swap_geometry needs to form the weights again, and the halo plan
    bool hasInterface = false;
    std::vector<int> hleft, hright;       // reference left / right cell of each face (boundary: nCell + f)
    std::vector<int> forder, ord;         // storage face -> reference face, storage cell -> reference cell
    std::vector<int> bfacePos;            // storage position of each reference boundary face
    std::vector<uint8_t> itfFace;         // 1 for each reference boundary face of an interface region
    int *haloSend = nullptr, *haloRecv = nullptr;   // storage indices (device)
    int nHaloSend = 0, nHaloRecv = 0;
    bool nsForwardDone = false, saForwardDone = false;   // a forward sweep waits for its backward sweep
};

namespace {

const char *kGeomNames[12] = {"xfn", "yfn", "zfn", "area", "xfc", "yfc", "zfc", "xcc", "ycc", "zcc", "vol", "skew"};

int fail(phx_ctx *ctx, int code, const std::string &msg)
{
    if (ctx) ctx->err = msg;
    return code;
}

#define PHX_CUDA(ctx, call)                                                                      \
    do {                                                                                         \
        cudaError_t e_ = (call);                                                                 \
        if (e_ != cudaSuccess)                                                                   \
            return fail(ctx, PHX_ERR_CUDA, std::string(#call " failed: ") + cudaGetErrorString(e_)); \
    } while (0)

template <class T>
int dalloc(phx_ctx *ctx, T **p, size_t n)
{
    void *v = nullptr;
    if (n == 0) n = 1;
    cudaError_t e = cudaMalloc(&v, n * sizeof(T));
    if (e != cudaSuccess) return fail(ctx, PHX_ERR_CUDA, std::string("cudaMalloc failed: ") + cudaGetErrorString(e));
    ctx->allocs.push_back(v);
    *p = static_cast<T *>(v);
    return PHX_OK;
}

template <class T>
int upload(phx_ctx *ctx, const T **dst, const std::vector<T> &src)
{
    T *d = nullptr;
    int rc = dalloc(ctx, &d, src.size());
    if (rc) return rc;
    if (!src.empty()) PHX_CUDA(ctx, cudaMemcpy(d, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice));
    *dst = d;
    return PHX_OK;
}

// ---------------------------------------------------------------------------
// Grid metrics, FP64, following the reference's UnstructGrid::ComputeMetrics
// for 3-D grids (API/Geometry/src/Geo_UnstructGrid.cpp:5695-5709):
//  faces  ComputeFaceCenterAreaNormal3DNew2 (:5911-6043): node-average
//         centre refined 4 times to the area-weighted fan centroid, normal
//         from the fan cross products of the final pass;
//  cells  ComputeCellCenterVol3DNew2 (:6545-6819): fan tetrahedra against the
//         node-average centre, centroid kept when inside all face planes,
//         ghost centres mirrored across the boundary face;
//  skew   SkewnessSummary (:2206-2330), degrees.
// ---------------------------------------------------------------------------
struct HostGrid {
    int nNode, nFace, nCell, nBFace;
    const double *x, *y, *z;
    std::vector<int> foff, f2n, left, right, coff, c2n;
};

// GG-node schedule (NSSolverUnstruct::ComputeNodeValue, NSSolverUnstruct.cpp:
// 4734-5080, with ModifyNodeValue :5083-5116).  Nodes are numbered in the order
// the storage-ordered cells first touch them.  Per storage node: its
// contributions in the reference's accumulation order (boundary nodes: the
// faces of solid-wall regions, then far-field regions, then other
// non-symmetry regions, each region's faces in face order, skipping nodes of a
// higher-priority boundary type; the other nodes, symmetry nodes included:
// the cells around them in cell order), each {storage cell, or storage
// boundary face with the sign bit set} with its FP64 1/distance weight, and
// the weight sum accumulated in the same order.  Per storage face: its nodes
// in the face's node order, for the face averages of the gradient.
struct NodeSchedule {
    std::vector<int> off, src, foff, fidx, nodeOf;
    std::vector<double> w, wsum;
};

static void node_schedule(const HostGrid &h, const phx_grid_desc *gd, const std::vector<double> *geom,
                          const std::vector<int> &ord, const std::vector<int> &rank, const std::vector<int> &fpos,
                          const std::vector<int> &forder, NodeSchedule &ns)
{
    const int nn = h.nNode, nc = h.nCell, nb = h.nBFace, nf = h.nFace;
    enum { kNoBC = -1 };
    std::vector<int> &nodeOf = ns.nodeOf;
    nodeOf.assign(nn, -1);
    int next = 0;
    for (int i = 0; i < nc; ++i) {
        const int c = ord[i];
        for (int j = h.coff[c]; j < h.coff[c + 1]; ++j)
            if (nodeOf[h.c2n[j]] < 0) nodeOf[h.c2n[j]] = next++;
    }
    for (int p = 0; p < nn; ++p)
        if (nodeOf[p] < 0) nodeOf[p] = next++;
    // node boundary types by priority: solid wall, far field, the other types but symmetry
    std::vector<std::vector<int>> rfaces((size_t)gd->n_region);
    for (int f = 0; f < nb; ++f) rfaces[gd->bface_region[f]].push_back(f);
    std::vector<int> nbc(nn, kNoBC);
    auto type = [&](int r) { return gd->region_type[r]; };
    for (int r = 0; r < gd->n_region; ++r)
        if (type(r) == PHX_BC_SOLID_SURFACE)
            for (int f : rfaces[r])
                for (int j = h.foff[f]; j < h.foff[f + 1]; ++j) nbc[h.f2n[j]] = PHX_BC_SOLID_SURFACE;
    for (int r = 0; r < gd->n_region; ++r)
        if (type(r) == PHX_BC_FARFIELD)
            for (int f : rfaces[r])
                for (int j = h.foff[f]; j < h.foff[f + 1]; ++j)
                    if (nbc[h.f2n[j]] != PHX_BC_SOLID_SURFACE) nbc[h.f2n[j]] = PHX_BC_FARFIELD;
    for (int r = 0; r < gd->n_region; ++r) {
        const int bt = type(r);
        if (bt == PHX_BC_SOLID_SURFACE || bt == PHX_BC_FARFIELD || bt == PHX_BC_SYMMETRY) continue;
        for (int f : rfaces[r])
            for (int j = h.foff[f]; j < h.foff[f + 1]; ++j) {
                const int p = h.f2n[j];
                if (nbc[p] != PHX_BC_SOLID_SURFACE && nbc[p] != PHX_BC_FARFIELD) nbc[p] = bt;
            }
    }
    const double *xfc = geom[4].data(), *yfc = geom[5].data(), *zfc = geom[6].data();
    const double *xcc = geom[7].data(), *ycc = geom[8].data(), *zcc = geom[9].data();
    // every contribution in the reference's order: emit(reference node, source, weight)
    auto visit = [&](auto &&emit) {
        for (int step = 1; step <= 3; ++step)
            for (int r = 0; r < gd->n_region; ++r) {
                const int bt = type(r);
                const bool take = step == 1 ? bt == PHX_BC_SOLID_SURFACE
                                : step == 2 ? bt == PHX_BC_FARFIELD
                                            : (bt != PHX_BC_SOLID_SURFACE && bt != PHX_BC_FARFIELD &&
                                               bt != PHX_BC_SYMMETRY);
                if (!take) continue;
                for (int f : rfaces[r])
                    for (int j = h.foff[f]; j < h.foff[f + 1]; ++j) {
                        const int p = h.f2n[j];
                        if (step == 2 && nbc[p] == PHX_BC_SOLID_SURFACE) continue;
                        if (step == 3 && (nbc[p] == PHX_BC_SOLID_SURFACE || nbc[p] == PHX_BC_FARFIELD)) continue;
                        const double dx = h.x[p] - xfc[f], dy = h.y[p] - yfc[f], dz = h.z[p] - zfc[f];
                        emit(p, (int)((unsigned)fpos[f] | 0x80000000u), 1.0 / std::sqrt(dx * dx + dy * dy + dz * dz));
                    }
            }
        for (int c = 0; c < nc; ++c)
            for (int j = h.coff[c]; j < h.coff[c + 1]; ++j) {
                const int p = h.c2n[j];
                if (nbc[p] != kNoBC) continue;
                const double dx = h.x[p] - xcc[c], dy = h.y[p] - ycc[c], dz = h.z[p] - zcc[c];
                emit(p, rank[c], 1.0 / std::sqrt(dx * dx + dy * dy + dz * dz));
            }
    };
    ns.off.assign(nn + 1, 0);
    visit([&](int p, int, double) { ns.off[nodeOf[p] + 1]++; });
    for (int i = 0; i < nn; ++i) ns.off[i + 1] += ns.off[i];
    ns.src.resize(ns.off[nn]);
    ns.w.resize(ns.off[nn]);
    ns.wsum.assign(nn, 0.0);
    std::vector<int> fill(ns.off.begin(), ns.off.end() - 1);
    visit([&](int p, int src, double wt) {
        const int i = nodeOf[p];
        ns.src[fill[i]] = src;
        ns.w[fill[i]++] = wt;
        ns.wsum[i] += wt;
    });
    ns.foff.assign(nf + 1, 0);
    for (int sf = 0; sf < nf; ++sf) {
        const int f = forder[sf];
        ns.foff[sf + 1] = ns.foff[sf] + (h.foff[f + 1] - h.foff[f]);
    }
    ns.fidx.resize(ns.foff[nf]);
    for (int sf = 0; sf < nf; ++sf) {
        const int f = forder[sf];
        for (int j = h.foff[f], k = ns.foff[sf]; j < h.foff[f + 1]; ++j, ++k) ns.fidx[k] = nodeOf[h.f2n[j]];
    }
}

// GG-node schedule of the SA variable (TurbSolverUnstr::ComputeQTurbNodeValue,
// TurbSolverUnstr.cpp:3480-3814, and ModifyQTurbNodeValue :3816-3845): every
// face adds its two sides' values to each of its nodes -- the boundary faces
// region by region with the face-to-node list read at a running position, as
// the reference reads it, then the interior faces -- and the nodes of
// symmetry, then far-field, then solid-wall faces are reset and take those
// faces only.  Per storage node: the pairs {storage owner, storage other
// side} in that order (the node value is their sum over twice their count).
struct TurbNodeSchedule {
    std::vector<int> off;
    std::vector<int2> pairs;
};

static void turb_node_schedule(const HostGrid &h, const phx_grid_desc *gd, const std::vector<int> &nodeOf,
                               const std::vector<int> &rank, const std::vector<int> &fpos, TurbNodeSchedule &ts)
{
    const int nn = h.nNode, nc = h.nCell, nb = h.nBFace, nf = h.nFace;
    std::vector<std::vector<int>> rfaces((size_t)gd->n_region);
    for (int f = 0; f < nb; ++f) rfaces[gd->bface_region[f]].push_back(f);
    // the running positions of the boundary faces' node blocks, regions in order
    std::vector<int> bpos(nb);
    int pos = 0;
    for (int r = 0; r < gd->n_region; ++r)
        for (int f : rfaces[r]) { bpos[f] = pos; pos += h.foff[f + 1] - h.foff[f]; }
    // the last reset that reaches each node: 0 none, 1 symmetry, 2 far field, 3 solid wall
    std::vector<uint8_t> cat(nn, 0);
    const int kinds[3] = {PHX_BC_SYMMETRY, PHX_BC_FARFIELD, PHX_BC_SOLID_SURFACE};
    for (int k = 0; k < 3; ++k)
        for (int r = 0; r < gd->n_region; ++r)
            if (gd->region_type[r] == kinds[k])
                for (int f : rfaces[r])
                    for (int j = 0; j < h.foff[f + 1] - h.foff[f]; ++j) cat[h.f2n[bpos[f] + j]] = (uint8_t)(k + 1);
    auto other = [&](int f) { return f < nb ? nc + fpos[f] : rank[h.right[f]]; };
    auto visit = [&](auto &&emit) {
        for (int r = 0; r < gd->n_region; ++r)   // boundary faces: nodes outside the three kinds keep these
            for (int f : rfaces[r])
                for (int j = 0; j < h.foff[f + 1] - h.foff[f]; ++j) {
                    const int p = h.f2n[bpos[f] + j];
                    if (cat[p] == 0) emit(p, rank[h.left[f]], other(f));
                }
        for (int f = nb; f < nf; ++f)
            for (int j = h.foff[f]; j < h.foff[f + 1]; ++j) {
                const int p = h.f2n[j];
                if (cat[p] == 0) emit(p, rank[h.left[f]], other(f));
            }
        for (int k = 0; k < 3; ++k)
            for (int r = 0; r < gd->n_region; ++r)
                if (gd->region_type[r] == kinds[k])
                    for (int f : rfaces[r])
                        for (int j = 0; j < h.foff[f + 1] - h.foff[f]; ++j) {
                            const int p = h.f2n[bpos[f] + j];
                            if (cat[p] == k + 1) emit(p, rank[h.left[f]], other(f));
                        }
    };
    ts.off.assign(nn + 1, 0);
    visit([&](int p, int, int) { ts.off[nodeOf[p] + 1]++; });
    for (int i = 0; i < nn; ++i) ts.off[i + 1] += ts.off[i];
    ts.pairs.resize(ts.off[nn]);
    std::vector<int> fill(ts.off.begin(), ts.off.end() - 1);
    visit([&](int p, int a, int b) { ts.pairs[fill[nodeOf[p]]++] = make_int2(a, b); });
}

void face_metrics(const HostGrid &h, std::vector<double> *G)
{
    double *xfn = G[0].data(), *yfn = G[1].data(), *zfn = G[2].data(), *area = G[3].data();
    double *xfc = G[4].data(), *yfc = G[5].data(), *zfc = G[6].data();
    for (int f = 0; f < h.nFace; ++f) {
        const int b = h.foff[f], nn = h.foff[f + 1] - b;
        double cx = 0, cy = 0, cz = 0;
        for (int j = 0; j < nn; ++j) {
            const int p = h.f2n[b + j];
            cx += h.x[p]; cy += h.y[p]; cz += h.z[p];
        }
        const double inv = 1.0 / nn;
        cx *= inv; cy *= inv; cz *= inv;
        double sx = 0, sy = 0, sz = 0;
        for (int pass = 0; pass < 5; ++pass) {
            double wx = 0, wy = 0, wz = 0, wa = 0;
            sx = sy = sz = 0;
            for (int j = 0; j < nn; ++j) {
                const int a1 = h.f2n[b + j], a2 = h.f2n[b + (j + 1) % nn];
                const double ux = h.x[a1] - cx, uy = h.y[a1] - cy, uz = h.z[a1] - cz;
                const double vx = h.x[a2] - cx, vy = h.y[a2] - cy, vz = h.z[a2] - cz;
                const double nx = uy * vz - vy * uz, ny = uz * vx - vz * ux, nz = ux * vy - vx * uy;
                const double ta = std::sqrt(nx * nx + ny * ny + nz * nz);
                wa += ta;
                wx += ta * (h.x[a1] + h.x[a2] + cx);
                wy += ta * (h.y[a1] + h.y[a2] + cy);
                wz += ta * (h.z[a1] + h.z[a2] + cz);
                sx += nx; sy += ny; sz += nz;
            }
            if (wa > kSmall) {
                const double t = 1.0 / wa / 3.0;
                cx = wx * t; cy = wy * t; cz = wz * t;
            }
        }
        const double s = std::sqrt(sx * sx + sy * sy + sz * sz);
        area[f] = s * 0.5;
        const double os = 1.0 / (s + kSmall);
        xfn[f] = sx * os; yfn[f] = sy * os; zfn[f] = sz * os;
        xfc[f] = cx; yfc[f] = cy; zfc[f] = cz;
    }
}

void cell_metrics(const HostGrid &h, std::vector<double> *G)
{
    const double *xfn = G[0].data(), *yfn = G[1].data(), *zfn = G[2].data(), *area = G[3].data();
    const double *xfc = G[4].data(), *yfc = G[5].data(), *zfc = G[6].data();
    double *xcc = G[7].data(), *ycc = G[8].data(), *zcc = G[9].data(), *vol = G[10].data();
    const int nc = h.nCell, nb = h.nBFace;
    for (int c = 0; c < nc; ++c) {
        const int b = h.coff[c], nn = h.coff[c + 1] - b;
        double sx = 0, sy = 0, sz = 0;
        for (int j = 0; j < nn; ++j) {
            const int p = h.c2n[b + j];
            sx += h.x[p]; sy += h.y[p]; sz += h.z[p];
        }
        xcc[c] = sx / nn; ycc[c] = sy / nn; zcc[c] = sz / nn;
    }
    std::vector<double> tx(nc, 0.0), ty(nc, 0.0), tz(nc, 0.0);
    std::fill(vol, vol + nc, 0.0);
    auto add_tet = [&](int c, int f, int p2, int p3, double nx, double ny, double nz, double sign) {
        const double dx = xcc[c] - xfc[f], dy = ycc[c] - yfc[f], dz = zcc[c] - zfc[f];
        double ex = xfc[f] + h.x[p2] + h.x[p3] + xcc[c];
        double ey = yfc[f] + h.y[p2] + h.y[p3] + ycc[c];
        double ez = zfc[f] + h.z[p2] + h.z[p3] + zcc[c];
        double t = nx * dx + ny * dy + nz * dz;
        if (sign < 0) t = -t;
        tx[c] += ex * t; ty[c] += ey * t; tz[c] += ez * t; vol[c] += t;
    };
    for (int f = 0; f < h.nFace; ++f) {
        const int b = h.foff[f], nn = h.foff[f + 1] - b;
        const int le = h.left[f], re = h.right[f];
        for (int j = 0; j < nn; ++j) {
            const int p2 = h.f2n[b + j], p3 = h.f2n[b + (j + 1) % nn];
            const double ax = h.x[p2] - xfc[f], ay = h.y[p2] - yfc[f], az = h.z[p2] - zfc[f];
            const double bx = h.x[p3] - xfc[f], by = h.y[p3] - yfc[f], bz = h.z[p3] - zfc[f];
            const double nx = ay * bz - by * az, ny = az * bx - bz * ax, nz = ax * by - bx * ay;
            add_tet(le, f, p2, p3, nx, ny, nz, -1.0);
            if (f >= nb) add_tet(re, f, p2, p3, nx, ny, nz, +1.0);
        }
    }
    for (int c = 0; c < nc; ++c) {
        const double t = 1.0 / (4.0 * vol[c] + kSmall);
        tx[c] *= t; ty[c] *= t; tz[c] *= t;
        vol[c] /= 6.0;
    }
    std::vector<char> inside(nc, 1);
    for (int f = 0; f < h.nFace; ++f) {
        const int le = h.left[f];
        if ((tx[le] - xfc[f]) * xfn[f] + (ty[le] - yfc[f]) * yfn[f] + (tz[le] - zfc[f]) * zfn[f] > 0.0) inside[le] = 0;
        if (f >= nb) {
            const int re = h.right[f];
            if ((tx[re] - xfc[f]) * xfn[f] + (ty[re] - yfc[f]) * yfn[f] + (tz[re] - zfc[f]) * zfn[f] < 0.0) inside[re] = 0;
        }
    }
    for (int c = 0; c < nc; ++c)
        if (inside[c]) { xcc[c] = tx[c]; ycc[c] = ty[c]; zcc[c] = tz[c]; }
    for (int f = 0; f < nb; ++f) {
        const int le = h.left[f], re = nc + f;
        if (area[f] > kSmall) {
            const double d = 2.0 * ((xcc[le] - xfc[f]) * xfn[f] + (ycc[le] - yfc[f]) * yfn[f] + (zcc[le] - zfc[f]) * zfn[f]);
            xcc[re] = xcc[le] - xfn[f] * d;
            ycc[re] = ycc[le] - yfn[f] * d;
            zcc[re] = zcc[le] - zfn[f] * d;
        } else {
            xcc[re] = -xcc[le] + 2.0 * xfc[f];
            ycc[re] = -ycc[le] + 2.0 * yfc[f];
            zcc[re] = -zcc[le] + 2.0 * zfc[f];
        }
        vol[re] = vol[le];
    }
}

double clampunit(double v) { return v > 1.0 ? 1.0 : (v < -1.0 ? -1.0 : v); }

void skewness(const HostGrid &h, std::vector<double> *G)
{
    const double *xfn = G[0].data(), *yfn = G[1].data(), *zfn = G[2].data(), *area = G[3].data();
    const double *xfc = G[4].data(), *yfc = G[5].data(), *zfc = G[6].data();
    const double *xcc = G[7].data(), *ycc = G[8].data(), *zcc = G[9].data();
    double *skew = G[11].data();
    const double pi = 3.141592653589793;
    std::fill(skew, skew + h.nCell, 180.0);
    auto angle_to = [&](int f, double dx, double dy, double dz) {
        const double d = std::sqrt(dx * dx + dy * dy + dz * dz);
        return std::asin(clampunit((xfn[f] * dx + yfn[f] * dy + zfn[f] * dz) / (d + kSmall)));
    };
    for (int f = h.nBFace; f < h.nFace; ++f) {
        if (area[f] <= kSmall) continue;
        const int le = h.left[f], re = h.right[f];
        const double a1 = angle_to(f, xfc[f] - xcc[le], yfc[f] - ycc[le], zfc[f] - zcc[le]);
        const double a2 = angle_to(f, xcc[re] - xfc[f], ycc[re] - yfc[f], zcc[re] - zfc[f]);
        const double ang = std::min(a1, a2) * 180.0 / pi;
        skew[le] = std::min(skew[le], ang);
        skew[re] = std::min(skew[re], ang);
    }
    for (int f = 0; f < h.nBFace; ++f) {
        if (area[f] <= kSmall) continue;
        const int le = h.left[f];
        skew[le] = std::min(skew[le], angle_to(f, xfc[f] - xcc[le], yfc[f] - ycc[le], zfc[f] - zcc[le]) * 180.0 / pi);
    }
}

}  // namespace


// ---------------------------------------------------------------------------
// Storage order: Morton code of the cell centroids (21 bits per axis over the
// bounding box), ties by reference number.
// ---------------------------------------------------------------------------
namespace {

uint64_t spread3(uint64_t v)
{
    v &= 0x1fffff;
    v = (v | v << 32) & 0x1f00000000ffffULL;
    v = (v | v << 16) & 0x1f0000ff0000ffULL;
    v = (v | v << 8) & 0x100f00f00f00f00fULL;
    v = (v | v << 4) & 0x10c30c30c30c30c3ULL;
    v = (v | v << 2) & 0x1249249249249249ULL;
    return v;
}

// Least-squares weights (UnstructGrid::ComputeWeight, Geo_UnstructGrid.cpp:3761-3935,
// 3-D, every face mark 1): per face the inverse squared centre distance (ghost
// centre for boundary faces), per cell the inverse of sum_f w d d^T, zeroed
// when its determinant is below SMALL.  Reference order; m6 is [nCell][6].
void lsq_weights(const HostGrid &h, const std::vector<double> *G, std::vector<double> &iwt, std::vector<double> &m6)
{
    const int nc = h.nCell, nb = h.nBFace, nf = h.nFace;
    const double *xcc = G[7].data(), *ycc = G[8].data(), *zcc = G[9].data();
    iwt.assign(nf, 0.0);
    m6.assign((size_t)nc * 6, 0.0);
    for (int f = 0; f < nf; ++f) {
        const int le = h.left[f], re = f < nb ? nc + f : h.right[f];
        const double dx = (xcc[re] - xcc[le]) * 1.0, dy = (ycc[re] - ycc[le]) * 1.0, dz = (zcc[re] - zcc[le]) * 1.0;
        const double ods = 1.0 / (dx * dx + dy * dy + dz * dz + kSmall);
        const double t[6] = {ods * dx * dx, ods * dy * dy, ods * dz * dz, ods * dx * dy, ods * dx * dz, ods * dy * dz};
        iwt[f] = ods;
        for (int k = 0; k < 6; ++k) m6[(size_t)le * 6 + k] += t[k];
        if (f >= nb)
            for (int k = 0; k < 6; ++k) m6[(size_t)re * 6 + k] += t[k];
    }
    for (int c = 0; c < nc; ++c) {
        double *m = &m6[(size_t)c * 6];
        const double txx = m[0], tyy = m[1], tzz = m[2], txy = m[3], txz = m[4], tyz = m[5];
        const double delt = (txx * tyy * tzz + 2.0 * txy * txz * tyz - txx * tyz * tyz - tyy * txz * txz - tzz * txy * txy);
        if (std::fabs(delt) < kSmall) {
            for (int k = 0; k < 6; ++k) m[k] = 0.0;
        } else {
            const double od = 1.0 / delt;
            m[0] = (tyy * tzz - tyz * tyz) * od;
            m[1] = (txx * tzz - txz * txz) * od;
            m[2] = (txx * tyy - txy * txy) * od;
            m[3] = (txz * tyz - txy * tzz) * od;
            m[4] = (txy * tyz - txz * tyy) * od;
            m[5] = (txy * txz - tyz * txx) * od;
        }
    }
}

// Geometry switches of ComputeVisflux (NSSolverUnstruct.cpp:13147-13236) per
// reference face: bit 0 when both centre angles exceed skewnessAngle, bit 1
// when both are positive and |dL|, |dR| > TINY; bit 2 for the SA diffusion
// (TurbSolverUnstr::ComputeVisflux, TurbSolverUnstr.cpp:4520-4530): both above
// turbSkewnessAngle and |dL|, |dR| > TINY.
std::vector<uint8_t> viscous_flags(const HostGrid &h, const std::vector<double> *G, double skewAngle,
                                   double turbSkewAngle)
{
    const int nc = h.nCell, nb = h.nBFace, nf = h.nFace;
    std::vector<uint8_t> vf(nf, 0);
    for (int f = 0; f < nf; ++f) {
        const int le = h.left[f], re = f < nb ? nc + f : h.right[f];
        const double nxs = G[0][f], nys = G[1][f], nzs = G[2][f];
        const double dxL = G[7][le] - G[4][f], dyL = G[8][le] - G[5][f], dzL = G[9][le] - G[6][f];
        const double dxR = G[7][re] - G[4][f], dyR = G[8][re] - G[5][f], dzR = G[9][re] - G[6][f];
        const double dL = nxs * dxL + nys * dyL + nzs * dzL;
        const double dR = nxs * dxR + nys * dyR + nzs * dzR;
        double t = -dL / (std::sqrt(dxL * dxL + dyL * dyL + dzL * dzL) + kSmall);
        t = std::min(t, 1.0);
        t = std::max(t, -1.0);
        const double a1 = std::asin(t) * 180.0 / 3.141592653589793;
        t = dR / (std::sqrt(dxR * dxR + dyR * dyR + dzR * dzR) + kSmall);
        t = std::min(t, 1.0);
        t = std::max(t, -1.0);
        const double a2 = std::asin(t) * 180.0 / 3.141592653589793;
        uint8_t b = 0;
        if (a1 > skewAngle && a2 > skewAngle) b |= 1;
        if (a1 > 0.0 && a2 > 0.0 && std::fabs(dL) > kSmall && std::fabs(dR) > kSmall) b |= 2;
        if (a1 > turbSkewAngle && a2 > turbSkewAngle && std::fabs(dL) > kSmall && std::fabs(dR) > kSmall) b |= 4;
        vf[f] = b;
    }
    return vf;
}

std::vector<int> morton_order(int n, const double *x, const double *y, const double *z)
{
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    const double *a[3] = {x, y, z};
    for (int d = 0; d < 3; ++d)
        for (int i = 0; i < n; ++i) { lo[d] = std::min(lo[d], a[d][i]); hi[d] = std::max(hi[d], a[d][i]); }
    std::vector<std::pair<uint64_t, int>> key(n);
    for (int i = 0; i < n; ++i) {
        uint64_t code = 0;
        for (int d = 0; d < 3; ++d) {
            const double span = hi[d] - lo[d];
            const double t = span > 0 ? (a[d][i] - lo[d]) / span : 0.0;
            const uint64_t q = (uint64_t)std::min(2097151.0, std::max(0.0, t * 2097151.0));
            code |= spread3(q) << d;
        }
        key[i] = {code, i};
    }
    std::sort(key.begin(), key.end());
    std::vector<int> ord(n);
    for (int i = 0; i < n; ++i) ord[i] = key[i].second;
    return ord;
}

// Reverse Cuthill-McKee order of the cells over their interior faces: from a
// pseudo-peripheral cell (the far end of a breadth-first search from a
// minimum-degree cell), breadth-first, each cell's unvisited neighbours in
// increasing degree, every connected component in turn, then reversed.
std::vector<int> rcm_order(int nc, int nb, const std::vector<int> &c2f_off, const std::vector<int> &c2f,
                           const std::vector<int> &left, const std::vector<int> &right)
{
    auto nbr = [&](int c, int j) {
        const int f = c2f[j];
        if (f < nb) return -1;
        return left[f] == c ? right[f] : left[f];
    };
    std::vector<int> deg(nc, 0);
    for (int c = 0; c < nc; ++c)
        for (int j = c2f_off[c]; j < c2f_off[c + 1]; ++j) deg[c] += nbr(c, j) >= 0;
    std::vector<int> ord;
    ord.reserve(nc);
    std::vector<int> mark(nc, 0);   // 0 unvisited; BFS stamps
    std::vector<int> q, tmp;
    q.reserve(nc);
    int stamp = 1;
    // breadth-first from s over unvisited cells (mark != final); returns the last cell reached
    auto far_end = [&](int s) {
        ++stamp;
        q.clear();
        q.push_back(s);
        mark[s] = stamp;
        size_t h = 0;
        int last = s;
        while (h < q.size()) {
            const int c = q[h++];
            last = c;
            for (int j = c2f_off[c]; j < c2f_off[c + 1]; ++j) {
                const int o = nbr(c, j);
                if (o >= 0 && mark[o] != -1 && mark[o] != stamp) { mark[o] = stamp; q.push_back(o); }
            }
        }
        return last;
    };
    std::vector<int> byDeg(nc);
    for (int c = 0; c < nc; ++c) byDeg[c] = c;
    std::stable_sort(byDeg.begin(), byDeg.end(), [&](int a, int b) { return deg[a] < deg[b]; });
    for (int start : byDeg) {
        if (mark[start] == -1) continue;
        const int s = far_end(far_end(start));   // two searches: a pseudo-peripheral cell
        const size_t first = ord.size();
        ord.push_back(s);
        mark[s] = -1;
        for (size_t h = first; h < ord.size(); ++h) {
            const int c = ord[h];
            tmp.clear();
            for (int j = c2f_off[c]; j < c2f_off[c + 1]; ++j) {
                const int o = nbr(c, j);
                if (o >= 0 && mark[o] != -1) { mark[o] = -1; tmp.push_back(o); }
            }
            std::stable_sort(tmp.begin(), tmp.end(), [&](int a, int b) { return deg[a] < deg[b]; });
            ord.insert(ord.end(), tmp.begin(), tmp.end());
        }
    }
    std::reverse(ord.begin(), ord.end());
    return ord;
}

double entropy_fix_coefficient(double mach, double scale)
{
    // Param_NSSolver::SetEntropyFixCoefficients, CFD/NSSolver/src/Param_NSSolver.cpp:224-268
    double e;
    if (mach <= 0.6) e = 0.0001;
    else if (mach <= 2.0) e = 0.0001 * (mach - 2.0) / (0.6 - 2.0) + 0.01 * (mach - 0.6) / (2.0 - 0.6);
    else if (mach <= 5.0) e = 0.01 * (mach - 5.0) / (2.0 - 5.0) + 0.5 * (mach - 2.0) / (5.0 - 2.0);
    else e = 1.0;
    return e * scale;
}

double total_pressure(double gama, double mach)
{
    // PerfectGas::ComputePTotal, API/Physics/src/PerfectGas.cpp:1609-1640 (NaN
    // for the subsonic Mach numbers where the base of the power is negative,
    // as in the reference; NaN switches the pressure-based CFL limit off)
    double p = 1.0 / (gama * mach * mach);
    const double m12 = mach * mach, gp1 = gama + 1.0, gm1 = gama - 1.0;
    const double c1 = 2.0 / gm1 + m12;
    const double c2 = 2.0 * gama / gm1 * m12 - 1.0;
    const double cc = gama / (gama - 1.0);
    const double t0t = 1.0 + 0.5 * gm1 * c1 / c2;
    if (mach > 1.0) p *= (2.0 * gama / gp1 * m12 - gm1 / gp1);
    return p * std::pow(t0t, cc);
}

bool limiter_zeroed(int bcType)
{
    // SetLimitBoundary, Geo_UnstructGrid.cpp:10744-10775 (interface faces are left alone, :10758)
    return bcType != PHX_BC_SYMMETRY && bcType != PHX_BC_SOLID_SURFACE && bcType != PHX_BC_OUTFLOW &&
           bcType != PHX_BC_INTERFACE;
}

// Viscosity record of a laminar run: eddy viscosity 0, laminar viscosity of the
// NS step (read by the wall forces).
template <class T>
int make_visc(phx_ctx *ctx, Work<T> &w)
{
    const size_t nt = ctx->nTotal;
    int r = dalloc(ctx, &w.trec, nt * kTr);
    if (r) return r;
    std::vector<T> rec(nt * kTr, T(0));
    for (size_t i = 0; i < nt; ++i) rec[i * kTr + 2] = T(1);
    PHX_CUDA(ctx, cudaMemcpy(w.trec, rec.data(), sizeof(T) * nt * kTr, cudaMemcpyHostToDevice));
    return PHX_OK;
}

// Spalart-Allmaras arrays: nu~ of the free stream everywhere (TurbSolverUnstr::
// InitFlowAsRestart, TurbSolverUnstr.cpp:910-930), eddy viscosity 0 and laminar
// viscosity 1 until the first NS step forms it (NSSolverUnstruct.cpp:685-695).
template <class T>
int make_turb(phx_ctx *ctx, Work<T> &w, TurbWork<T> &t)
{
    const size_t nt = ctx->nTotal, nc = ctx->nCell, nf = ctx->nFace;
    int r = 0;
    r |= dalloc(ctx, &w.trec, nt * kTr);
    r |= dalloc(ctx, &t.qt64, nt);
    r |= dalloc(ctx, &t.tgrad, nc * kTg);
    r |= dalloc(ctx, &t.tcrec, nc * kTc);
    r |= dalloc(ctx, &t.tface, nf * kTf);
    r |= dalloc(ctx, &t.tcoef, 2 * nf);
    r |= dalloc(ctx, &t.tdq, nc);
    r |= dalloc(ctx, &t.tdqf, nc);
    r |= dalloc(ctx, &t.tdfl, nc);
    r |= dalloc(ctx, &t.tsrc, nc);
    if (ctx->prm.gradientName == 2) r |= dalloc(ctx, &t.qtnode, (size_t)ctx->nNode);
    r |= dalloc(ctx, &ctx->nmlp, 1);
    r |= dalloc(ctx, &ctx->mlpW, (size_t)kMlpH * kMlpK1 + 2 * (size_t)kMlpH * kMlpH);
    r |= dalloc(ctx, &ctx->mlpF, 4 * (size_t)kMlpH);
    r |= dalloc(ctx, &ctx->mlpOcc, (size_t)kMlpGrid * kMlpGrid);
    if (r) return r;
    PHX_CUDA(ctx, cudaMemset(ctx->nmlp, 0, sizeof(unsigned long long)));
    const double nu = ctx->nc.nutInf;
    std::vector<double> q(nt, nu);
    std::vector<T> rec(nt * kTr);
    for (size_t i = 0; i < nt; ++i) {
        rec[i * kTr] = (T)nu;
        rec[i * kTr + 1] = T(0);
        rec[i * kTr + 2] = T(1);
        rec[i * kTr + 3] = T(0);
    }
    PHX_CUDA(ctx, cudaMemcpy(t.qt64, q.data(), sizeof(double) * nt, cudaMemcpyHostToDevice));
    PHX_CUDA(ctx, cudaMemcpy(w.trec, rec.data(), sizeof(T) * nt * kTr, cudaMemcpyHostToDevice));
    PHX_CUDA(ctx, cudaMemset(t.tcoef, 0, sizeof(T) * 2 * nf));
    return PHX_OK;
}

template <class T>
int make_work(phx_ctx *ctx, Work<T> &w, const std::vector<double> &limInit)
{
    const size_t nt = ctx->nTotal, nc = ctx->nCell, nf = ctx->nFace;
    int r = 0;
    r |= dalloc(ctx, &w.qrec, nt * kQ);
    r |= dalloc(ctx, &w.grec, nt * kG);
    r |= dalloc(ctx, &w.flux, nf * kFlux);
    r |= dalloc(ctx, &w.coef, 2 * nf * kCoef);
    r |= dalloc(ctx, &w.crec, nc * kC);
    r |= dalloc(ctx, &w.dtraw, nc);
    r |= dalloc(ctx, &w.dqrec, nt * kD);
    r |= dalloc(ctx, &w.dqfwd, nt * kD);
    r |= dalloc(ctx, &w.dflux, nc * kD);
    if (ctx->prm.gradientName == 2) r |= dalloc(ctx, &w.nrec, (size_t)ctx->nNode * kN);
    if (r) return r;
    if (w.nrec) PHX_CUDA(ctx, cudaMemset(w.nrec, 0, sizeof(T) * (size_t)ctx->nNode * kN));
    std::vector<T> q(nt * kQ, T(0));
    for (size_t i = 0; i < nt; ++i) q[i * kQ + 7] = (T)limInit[i];
    PHX_CUDA(ctx, cudaMemcpy(w.qrec, q.data(), sizeof(T) * q.size(), cudaMemcpyHostToDevice));
    PHX_CUDA(ctx, cudaMemset(w.dqrec, 0, sizeof(T) * nt * kD));
    PHX_CUDA(ctx, cudaMemset(w.dqfwd, 0, sizeof(T) * nt * kD));   // interface ghost rows until the first exchange
    PHX_CUDA(ctx, cudaMemset(w.grec, 0, sizeof(T) * nt * kG));
    PHX_CUDA(ctx, cudaMemset(w.crec, 0, sizeof(T) * nc * kC));
    PHX_CUDA(ctx, cudaMemset(w.coef, 0, sizeof(T) * 2 * nf * kCoef));
    return PHX_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

void phx_default_params(phx_params *p)
{
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    // defaults of PHengLEI/examples/bin/cfd_para.hypara
    p->precision = PHX_FP64;
    p->refGama = 1.4;
    p->refMachNumber = 0.73;
    p->attackd = 2.79;
    p->angleSlide = 0.0;
    p->viscousType = 3;
    p->refReNumber = 6.5e6;
    p->refDimensionalTemperature = 288.15;
    p->prl = 0.72;
    p->prt = 0.90;
    p->tsuth = 110.4;
    p->wallTemperature = -1.0;
    p->gradientName = 0;
    p->uns_limiter_name = 1;
    p->ivencat = 7;
    p->venkatCoeff = 5.0;
    p->reconmeth = 1;
    p->uns_scheme_name = 0;
    p->roeEntropyFixMethod = 3;
    p->roeEntropyScale = 1.0;
    p->CFLStart = 0.01;
    p->CFLEnd = 10.0;
    p->CFLVaryStep = 500;
    p->ktmax = 1.0e10;
    p->nLUSGSSweeps = 1;
    p->LUSGSTolerance = 0.01;
    p->skewnessAngle = 60.0;
    p->muoo = 3.0;
    p->turbCFLScale = 1.0;
    p->sa_source = 0;
    p->turbSkewnessAngle = 0.0;
    p->freeStreamViscosity = 1.0e-3;
    p->AusmpwPlusLimiter = 1.0;
    p->flowInitStep = 100;   // cfd_para.hypara:1290
    p->flowInitMethod = 0;
}

int phx_ctx_create(const phx_grid_desc *gd, const phx_params *prm, phx_ctx **out)
{
    if (!out) return PHX_ERR_ARG;
    *out = nullptr;
    if (!gd || !prm || !gd->x || !gd->y || !gd->z || !gd->face_nnode || !gd->face2node || !gd->left_cell ||
        !gd->right_cell || !gd->cell_nnode || !gd->cell2node || !gd->region_type || (gd->n_bface > 0 && !gd->bface_region))
        return PHX_ERR_ARG;
    if (gd->n_cell <= 0 || gd->n_face <= 0 || gd->n_bface < 0 || gd->n_bface > gd->n_face || gd->n_node <= 0 ||
        gd->n_cell + gd->n_bface > 0x3fffffffLL || gd->n_face > 0x3fffffffLL)
        return PHX_ERR_ARG;
    if (prm->precision != PHX_FP64 && prm->precision != PHX_MIXED) return PHX_ERR_ARG;
    // inviscid, laminar and Spalart-Allmaras; adiabatic walls (wallTemperature <= 0);
    // SA needs the wall distance of every cell
    if (prm->viscousType != 0 && prm->viscousType != 1 && prm->viscousType != 3) return PHX_ERR_ARG;
    if (prm->viscousType != 0 && (prm->wallTemperature > 0.0 || prm->refReNumber <= 0.0)) return PHX_ERR_ARG;
    if (prm->viscousType == 3 && (!gd->wall_dist || prm->sa_source < 0 || prm->sa_source > 2 ||
                                  prm->turbCFLScale <= 0.0))
        return PHX_ERR_ARG;
    // gradientName 0 ggcell, 1 lsq, 2 ggnode
    if (prm->gradientName < 0 || prm->gradientName > 2 ||
        prm->uns_scheme_name < PHX_SCHEME_ROE || prm->uns_scheme_name > PHX_SCHEME_VANLEER_ROTATE ||
        prm->roeEntropyFixMethod != 3 || prm->flowInitStep < 0 ||
        prm->uns_limiter_name < PHX_LIMITER_NOLIM || prm->uns_limiter_name > PHX_LIMITER_BARTH ||
        (prm->flowInitMethod != 0 && prm->flowInitMethod != 2) ||
        prm->nLUSGSSweeps != 1 || (prm->uns_limiter_name == 1 && prm->ivencat != 7))
        return PHX_ERR_ARG;

    phx_ctx *ctx = new phx_ctx();
    ctx->prm = *prm;
    ctx->mixed = prm->precision == PHX_MIXED;
    ctx->sa = prm->viscousType == 3;
    cudaGetDevice(&ctx->device);
    cudaDeviceGetAttribute(&ctx->numSMs, cudaDevAttrMultiProcessorCount, ctx->device);

    HostGrid h;
    h.nNode = (int)gd->n_node; h.nFace = (int)gd->n_face; h.nCell = (int)gd->n_cell; h.nBFace = (int)gd->n_bface;
    h.x = gd->x; h.y = gd->y; h.z = gd->z;
    const int nc = h.nCell, nb = h.nBFace, nf = h.nFace, nt = nc + nb;
    ctx->nNode = h.nNode; ctx->nFace = nf; ctx->nCell = nc; ctx->nBFace = nb; ctx->nTotal = nt;
    h.foff.resize(nf + 1);
    h.foff[0] = 0;
    for (int f = 0; f < nf; ++f) {
        if (gd->face_nnode[f] < 3) { delete ctx; return PHX_ERR_ARG; }
        h.foff[f + 1] = h.foff[f] + gd->face_nnode[f];
    }
    h.f2n.assign(gd->face2node, gd->face2node + h.foff[nf]);
    h.left.assign(gd->left_cell, gd->left_cell + nf);
    h.right.assign(gd->right_cell, gd->right_cell + nf);
    for (int f = 0; f < nb; ++f) h.right[f] = nc + f;
    for (int f = 0; f < nf; ++f)
        if (h.left[f] < 0 || h.left[f] >= nc || (f >= nb && (h.right[f] < 0 || h.right[f] >= nc))) {
            delete ctx;
            return PHX_ERR_ARG;
        }
    for (int i = 0; i < h.foff[nf]; ++i)
        if (h.f2n[i] < 0 || h.f2n[i] >= h.nNode) { delete ctx; return PHX_ERR_ARG; }
    h.coff.resize(nc + 1);
    h.coff[0] = 0;
    for (int c = 0; c < nc; ++c) {
        if (gd->cell_nnode[c] < 4) { delete ctx; return PHX_ERR_ARG; }
        h.coff[c + 1] = h.coff[c] + gd->cell_nnode[c];
    }
    h.c2n.assign(gd->cell2node, gd->cell2node + h.coff[nc]);
    for (int i = 0; i < h.coff[nc]; ++i)
        if (h.c2n[i] < 0 || h.c2n[i] >= h.nNode) { delete ctx; return PHX_ERR_ARG; }
    for (int f = 0; f < nb; ++f)
        if (gd->bface_region[f] < 0 || gd->bface_region[f] >= gd->n_region) { delete ctx; return PHX_ERR_ARG; }

    // FP64 metrics in the reference's order
    for (int k = 0; k < 7; ++k) ctx->geom[k].assign(nf, 0.0);
    for (int k = 7; k < 11; ++k) ctx->geom[k].assign(nt, 0.0);
    ctx->geom[11].assign(nc, 0.0);
    face_metrics(h, ctx->geom);
    cell_metrics(h, ctx->geom);
    skewness(h, ctx->geom);
    double vsum = 0.0;
    for (int c = 0; c < nc; ++c) vsum += ctx->geom[10][c];
    const double avgVol = vsum / (double)nc;   // Region::ComputeGlobalGridSize, Region.cpp:2655-2734

    // cell -> face lists in the reference's face order (UnstructGrid::ComputeCell2Face, :1246-1290)
    std::vector<int> c2f_off(nc + 1, 0), c2f;
    for (int f = 0; f < nf; ++f) { c2f_off[h.left[f] + 1]++; if (f >= nb) c2f_off[h.right[f] + 1]++; }
    for (int c = 0; c < nc; ++c) c2f_off[c + 1] += c2f_off[c];
    c2f.resize(c2f_off[nc]);
    {
        std::vector<int> fill(c2f_off.begin(), c2f_off.end() - 1);
        for (int f = 0; f < nf; ++f) { c2f[fill[h.left[f]]++] = f; if (f >= nb) c2f[fill[h.right[f]]++] = f; }
    }
    for (int c = 0; c < nc; ++c)
        if (c2f_off[c + 1] - c2f_off[c] > kSweepMaxEntries) { delete ctx; return PHX_ERR_ARG; }  // two sweep slots

    // storage order
    // storage order: Morton (Z-curve) order of the cell centres, or, with
    // PHX_CELL_ORDER=rcm, reverse Cuthill-McKee over the faces
    const char *co = getenv("PHX_CELL_ORDER");
    const std::vector<int> ord = (co && std::strcmp(co, "rcm") == 0)
                                     ? rcm_order(nc, nb, c2f_off, c2f, h.left, h.right)
                                     : morton_order(nc, ctx->geom[7].data(), ctx->geom[8].data(), ctx->geom[9].data());
    std::vector<int> rank(nc);
    for (int i = 0; i < nc; ++i) rank[ord[i]] = i;
    ctx->rankOf = rank;
    std::vector<int> forder(nf);   // storage face -> reference face
    for (int f = 0; f < nf; ++f) forder[f] = f;
    std::stable_sort(forder.begin(), forder.begin() + nb, [&](int a, int b) { return rank[h.left[a]] < rank[h.left[b]]; });
    std::stable_sort(forder.begin() + nb, forder.end(), [&](int a, int b) {
        const int ma = std::min(rank[h.left[a]], rank[h.right[a]]), mb = std::min(rank[h.left[b]], rank[h.right[b]]);
        if (ma != mb) return ma < mb;
        return std::max(rank[h.left[a]], rank[h.right[a]]) < std::max(rank[h.left[b]], rank[h.right[b]]);
    });
    std::vector<int> fpos(nf);
    for (int i = 0; i < nf; ++i) fpos[forder[i]] = i;
    // storage index of any reference cell or ghost (ghost of reference boundary face f: nc + f)
    auto sidx = [&](int c) { return c < nc ? rank[c] : nc + fpos[c - nc]; };

    // LU-SGS level schedules from the reference's cell numbers, with each
    // cell's entry count (neighbours on the sweep's side; the backward sweep
    // also reads the ghosts of the cell's boundary faces)
    std::vector<int> lev(nc, 0), cntF(nc, 0), cntB(nc, 0);
    int nfl = 0;
    for (int c = 0; c < nc; ++c) {
        int l = 0;
        for (int j = c2f_off[c]; j < c2f_off[c + 1]; ++j) {
            const int f = c2f[j];
            if (f < nb) { cntB[c]++; continue; }
            const int o = h.left[f] == c ? h.right[f] : h.left[f];
            if (o < c) { l = std::max(l, lev[o] + 1); cntF[c]++; }
            else cntB[c]++;
        }
        lev[c] = l;
        nfl = std::max(nfl, l + 1);
    }
    // Positions are slots of kSweepLanes lanes.  A cell with more entries
    // than one slot holds takes two adjacent slots (the second continues its
    // entries).  In each level the two-slot cells come first, so their slot
    // pairs start at even slot numbers and never straddle a warp, and each
    // level is padded with idle slots (-1) to a multiple of kSweepSlots, the
    // slots of one warp, so that the slots one warp takes together always lie
    // in one level and never depend on each other.
    auto bucket = [&](int nlev, const std::vector<int> &cnt, std::vector<int> &cells, std::vector<uint8_t> &cont,
                      bool ascending) {
        std::vector<int> nbig(nlev, 0), nsmall(nlev, 0), off(nlev + 1, 0);
        for (int c = 0; c < nc; ++c) (cnt[c] > kSweepLanes ? nbig : nsmall)[lev[c]]++;
        for (int l = 0; l < nlev; ++l)
            off[l + 1] = off[l] + (2 * nbig[l] + nsmall[l] + kSweepSlots - 1) / kSweepSlots * kSweepSlots;
        cells.assign(off[nlev], -1);
        cont.assign(off[nlev], 0);
        std::vector<int> fbig(off.begin(), off.end() - 1), fsmall(nlev);
        for (int l = 0; l < nlev; ++l) fsmall[l] = off[l] + 2 * nbig[l];
        auto put = [&](int c) {
            const int l = lev[c];
            if (cnt[c] > kSweepLanes) {
                cells[fbig[l]] = c;
                cells[fbig[l] + 1] = c;
                cont[fbig[l] + 1] = 1;
                fbig[l] += 2;
            } else {
                cells[fsmall[l]++] = c;
            }
        };
        if (ascending) for (int c = 0; c < nc; ++c) put(c);
        else for (int c = nc - 1; c >= 0; --c) put(c);
    };
    std::vector<int> fwd_cells, bwd_cells;
    std::vector<uint8_t> fwd_cont, bwd_cont;
    bucket(nfl, cntF, fwd_cells, fwd_cont, true);
    std::fill(lev.begin(), lev.end(), 0);
    int nbl = 0;
    for (int c = nc - 1; c >= 0; --c) {
        int l = 0;
        for (int j = c2f_off[c]; j < c2f_off[c + 1]; ++j) {
            const int f = c2f[j];
            if (f < nb) continue;
            const int o = h.left[f] == c ? h.right[f] : h.left[f];
            if (o > c) l = std::max(l, lev[o] + 1);
        }
        lev[c] = l;
        nbl = std::max(nbl, l + 1);
    }
    bucket(nbl, cntB, bwd_cells, bwd_cont, false);

    // sweep entries (storage indices) of each cell in the cell's face order:
    // {neighbour, face (sign bit set when the normal points into the cell),
    // index of the face use's factors (2 f + side), 0}
    auto cell_entries = [&](int c, bool forward, std::vector<int4> &e) {
        e.clear();
        for (int j = c2f_off[c]; j < c2f_off[c + 1]; ++j) {
            const int f = c2f[j];
            int nbr = -1;
            bool isLeft = true;
            if (f < nb) {
                if (!forward) nbr = nc + f;
            } else {
                isLeft = h.left[f] == c;
                const int o = isLeft ? h.right[f] : h.left[f];
                if (forward ? (o < c) : (o > c)) nbr = o;
            }
            if (nbr < 0) continue;
            e.push_back(make_int4(sidx(nbr), isLeft ? fpos[f] : (int)((unsigned)fpos[f] | 0x80000000u),
                                  2 * fpos[f] + (isLeft ? 0 : 1), 0));
        }
    };
    // per slot {storage cell, entry count} ({cell, -1} on the second slot of a
    // two-slot cell) and kSweepLanes entries (neighbour -1 on unused lanes), so
    // a lane reads its entry with one load and no offset lookup
    auto pack = [&](const std::vector<int> &cells, const std::vector<uint8_t> &cont, bool forward,
                    std::vector<int2> &pinfo, std::vector<int4> &ent) {
        const size_t npos = cells.size();
        pinfo.resize(npos);
        ent.assign(npos * kSweepLanes, make_int4(-1, 0, 0, 0));
        std::vector<int4> e;
        for (size_t i = 0; i < npos; ++i) {
            const int c = cells[i];
            if (c < 0) { pinfo[i] = make_int2(-1, 0); continue; }
            cell_entries(c, forward, e);
            const int n = (int)e.size();
            pinfo[i] = make_int2(rank[c], cont[i] ? -1 : n);
            const int k0 = cont[i] ? kSweepLanes : 0;
            for (int k = k0; k < std::min(n, k0 + kSweepLanes); ++k) ent[i * kSweepLanes + (k - k0)] = e[k];
        }
    };
    std::vector<int2> fwd_pinfo, bwd_pinfo;
    std::vector<int4> fwd_ent, bwd_ent;
    pack(fwd_cells, fwd_cont, true, fwd_pinfo, fwd_ent);
    pack(bwd_cells, bwd_cont, false, bwd_pinfo, bwd_ent);

    // boundary classification (storage face order)
    std::vector<int32_t> bkind(nb), btype(nb);
    std::vector<uint8_t> ffadj(nc, 0);
    std::vector<double> limInit(nt, 1.0);
    for (int fs = 0; fs < nb; ++fs) {
        const int f = forder[fs];
        const int t = gd->region_type[gd->bface_region[f]];
        btype[fs] = t;
        if (t == PHX_BC_SOLID_SURFACE) bkind[fs] = prm->viscousType ? BK_WALL : BK_SYMMETRY;
        else if (t == PHX_BC_SYMMETRY) bkind[fs] = BK_SYMMETRY;
        else if (t == PHX_BC_FARFIELD) bkind[fs] = BK_FARFIELD;
        else if (t == PHX_BC_INTERFACE) bkind[fs] = BK_INTERFACE;
        else { delete ctx; return PHX_ERR_ARG; }
        // SetLimitBoundary zeroes the far-field ghosts' limiter only when a limiter
        // runs; with nolim every limit2D entry is 1 (ComputeLimiter :18213-18220)
        if (limiter_zeroed(t)) {
            ffadj[rank[h.left[f]]] = 1;
            if (prm->uns_limiter_name == PHX_LIMITER_VENCAT || prm->uns_limiter_name == PHX_LIMITER_BARTH)
                limInit[nc + fs] = 0.0;
        }
    }

    // GG-node across zones needs the interpoint exchange of node values and
    // weights (Controller::PostSolve, Controller.cpp:5063-5205), which is not built
    ctx->hasInterface = std::find(bkind.begin(), bkind.end(), (int32_t)BK_INTERFACE) != bkind.end();
    if (ctx->hasInterface && prm->gradientName == 2) { delete ctx; return PHX_ERR_ARG; }

    std::vector<double> iwt, m6;
    if (prm->gradientName == 1) lsq_weights(h, ctx->geom, iwt, m6);

    // records in storage order
    std::vector<int2> lr(nf);
    std::vector<double> frec((size_t)nf * kF), xrec((size_t)nt * kX);
    for (int fs = 0; fs < nf; ++fs) {
        const int f = forder[fs];
        lr[fs] = make_int2(rank[h.left[f]], f < nb ? nc + fs : rank[h.right[f]]);
        for (int k = 0; k < 7; ++k) frec[(size_t)fs * kF + k] = ctx->geom[k][f];
        frec[(size_t)fs * kF + 7] = prm->gradientName == 1 ? iwt[f] : 0.0;
    }
    std::vector<uint8_t> vflag(nf, 0);
    if (prm->viscousType) {
        const std::vector<uint8_t> vref = viscous_flags(h, ctx->geom, prm->skewnessAngle, prm->turbSkewnessAngle);
        for (int fs = 0; fs < nf; ++fs) vflag[fs] = vref[forder[fs]];
    }
    std::vector<double> lsqs(prm->gradientName == 1 ? (size_t)nc * 8 : 8, 0.0);
    if (prm->gradientName == 1)
        for (int i = 0; i < nc; ++i)
            for (int k = 0; k < 6; ++k) lsqs[(size_t)i * 8 + k] = m6[(size_t)ord[i] * 6 + k];
    std::vector<int> origv(nt);
    for (int i = 0; i < nt; ++i) {
        const int c = i < nc ? ord[i] : nc + forder[i - nc];
        origv[i] = c;
        for (int k = 0; k < 4; ++k) xrec[(size_t)i * kX + k] = ctx->geom[7 + k][c];
    }
    std::vector<double> skew(nc), volpow(nc);
    for (int i = 0; i < nc; ++i) {
        skew[i] = ctx->geom[11][ord[i]];
        volpow[i] = std::pow(std::pow(ctx->geom[10][ord[i]], 1.0 / 3.0), 3.0);
    }
    std::vector<int> sc2f_off(nc + 1, 0), sc2f(c2f.size());
    for (int i = 0; i < nc; ++i) sc2f_off[i + 1] = sc2f_off[i] + (c2f_off[ord[i] + 1] - c2f_off[ord[i]]);
    for (int i = 0; i < nc; ++i) {
        const int c = ord[i];
        for (int j = c2f_off[c], k = sc2f_off[i]; j < c2f_off[c + 1]; ++j, ++k) sc2f[k] = fpos[c2f[j]];
    }

    // constants
    NsConst &k = ctx->nc;
    k.gama = prm->refGama;
    k.coefState = 1.0 / (prm->refGama * prm->refMachNumber * prm->refMachNumber);
    k.pTotal = total_pressure(prm->refGama, prm->refMachNumber);
    const double dr = 3.141592653589793 / 180.0;
    const double att = prm->attackd * dr, sid = prm->angleSlide * dr;
    k.primInf[0] = 1.0;
    k.primInf[1] = std::cos(att) * std::cos(sid);
    k.primInf[2] = std::sin(att) * std::cos(sid);
    k.primInf[3] = std::sin(sid);
    k.primInf[4] = k.coefState;
    k.acoustic = k.convective = entropy_fix_coefficient(prm->refMachNumber, prm->roeEntropyScale);
    k.scheme = prm->uns_scheme_name;
    k.ausmpwLim = prm->AusmpwPlusLimiter;
    const double K = prm->venkatCoeff;
    double kt = K * K * K;
    kt *= 1.0 / std::pow(std::pow(avgVol, 1.0 / 3.0), 3.0);
    k.venkatK3 = kt;
    k.viscous = prm->viscousType;
    k.limiter = prm->uns_limiter_name;
    k.reconMethod = prm->reconmeth;
    k.cflStart = prm->CFLStart; k.cflEnd = prm->CFLEnd; k.cflVaryStep = prm->CFLVaryStep;
    k.ktmax = prm->ktmax;
    k.nSweeps = prm->nLUSGSSweeps;
    k.lusgsTol = prm->LUSGSTolerance;
    k.reynolds = prm->refReNumber;
    k.gradient = prm->gradientName;
    // Param_NSSolverUnstruct getters; the Sutherland constant (110.4 K) over the
    // reference temperature (PerfectGas::ComputeReferenceViscosityDimensional,
    // PerfectGas.cpp:1486-1494)
    k.oRe = prm->viscousType ? 1.0 / prm->refReNumber : 0.0;
    k.oPrl = 1.0 / prm->prl;
    k.oPrt = 1.0 / prm->prt;
    k.cp = 1.0 / ((prm->refGama - 1.0) * (prm->refMachNumber * prm->refMachNumber));
    k.tsuth = prm->tsuth / prm->refDimensionalTemperature;
    k.skewAngle = prm->skewnessAngle;
    // Param_TurbSolver::Init (CFD/TurbSolver/src/Param_TurbSolver.cpp:249-256):
    // nu~ of the free stream = muoo / (rho_inf * turb_cmu + SMALL), turb_cmu = 1
    k.nutInf = prm->muoo / (k.primInf[0] * 1.0 + kSmall);
    k.vistInf = prm->freeStreamViscosity;
    k.turbCflScale = prm->turbCFLScale;
    k.saSource = prm->viscousType == 3 ? prm->sa_source : 0;
    k.spinLimit = kDefaultSpinLimit;
    k.holdCell = -1;

    // device grid
    DevGrid &g = ctx->g;
    g.nCell = nc; g.nBFace = nb; g.nFace = nf; g.nTotal = nt;
    g.avgVol = avgVol;
    g.nFwdLevels = nfl; g.nBwdLevels = nbl;
    g.nFwdPos = (int)fwd_cells.size(); g.nBwdPos = (int)bwd_cells.size();
    g.walldist = nullptr;
    int rc = 0;
    if (ctx->sa) {
        std::vector<double> wd(nc);
        for (int i = 0; i < nc; ++i) wd[i] = gd->wall_dist[ord[i]];
        rc |= upload(ctx, &g.walldist, wd);
    }
    rc |= upload(ctx, &g.lr, lr);
    rc |= upload(ctx, &g.frec, frec);
    rc |= upload(ctx, &g.vflag, vflag);
    rc |= upload(ctx, &g.lsq, lsqs);
    rc |= upload(ctx, &g.xrec, xrec);
    rc |= upload(ctx, &g.skew, skew);
    rc |= upload(ctx, &g.volpow, volpow);
    rc |= upload(ctx, &g.c2f_off, sc2f_off);
    rc |= upload(ctx, &g.c2f, sc2f);
    rc |= upload(ctx, &g.orig, origv);
    rc |= upload(ctx, &g.bkind, bkind);
    rc |= upload(ctx, &g.btype, btype);
    rc |= upload(ctx, &g.farfield_adj, ffadj);
    g.nNode = h.nNode;
    if (prm->gradientName == 2) {
        NodeSchedule ns;
        node_schedule(h, gd, ctx->geom, ord, rank, fpos, forder, ns);
        rc |= upload(ctx, &g.node_off, ns.off);
        rc |= upload(ctx, &g.node_src, ns.src);
        rc |= upload(ctx, &g.node_w, ns.w);
        rc |= upload(ctx, &g.node_wsum, ns.wsum);
        rc |= upload(ctx, &g.fn_off, ns.foff);
        rc |= upload(ctx, &g.fn_idx, ns.fidx);
        if (ctx->sa) {
            TurbNodeSchedule ts;
            turb_node_schedule(h, gd, ns.nodeOf, rank, fpos, ts);
            rc |= upload(ctx, &g.tn_off, ts.off);
            rc |= upload(ctx, &g.tn_pairs, ts.pairs);
        }
    }
    rc |= upload(ctx, &g.fwd_pinfo, fwd_pinfo);
    rc |= upload(ctx, &g.fwd_ent, fwd_ent);
    rc |= upload(ctx, &g.bwd_pinfo, bwd_pinfo);
    rc |= upload(ctx, &g.bwd_ent, bwd_ent);
    rc |= dalloc(ctx, &ctx->q64[0], (size_t)5 * nt);
    rc |= dalloc(ctx, &ctx->q64[1], (size_t)5 * nt);
    rc |= dalloc(ctx, &ctx->tmp, (size_t)5 * nt);
    rc |= dalloc(ctx, &ctx->red, 1);
    rc |= dalloc(ctx, &ctx->neglist, 1 << 16);
    if (!rc) rc = ctx->mixed ? make_work(ctx, ctx->w32, limInit) : make_work(ctx, ctx->w64, limInit);
    if (!rc && ctx->sa) rc = ctx->mixed ? make_turb(ctx, ctx->w32, ctx->t32) : make_turb(ctx, ctx->w64, ctx->t64);
    else if (!rc && prm->viscousType) rc = ctx->mixed ? make_visc(ctx, ctx->w32) : make_visc(ctx, ctx->w64);
    if (!rc) rc = dalloc(ctx, &ctx->forces, 16);
    if (!rc && cudaMemset(ctx->red, 0, sizeof(Reduce)) != cudaSuccess) rc = PHX_ERR_CUDA;
    if (rc) {
        const int code = rc < 0 ? rc : PHX_ERR_CUDA;
        phx_ctx_destroy(ctx);
        return code;
    }
    if (ctx->hasInterface) {
        ctx->hleft = h.left;
        ctx->hright = h.right;
        ctx->forder = forder;
        ctx->ord = ord;
        ctx->bfacePos.assign(fpos.begin(), fpos.begin() + nb);
        ctx->itfFace.assign(nb, 0);
        for (int fs = 0; fs < nb; ++fs) ctx->itfFace[forder[fs]] = bkind[fs] == BK_INTERFACE;
    }
    // free-stream initial state (NSSolverUnstruct::InitFlow), ghosts included
    std::vector<double> q0((size_t)5 * nt);
    for (int m = 0; m < 5; ++m) std::fill(q0.begin() + (size_t)m * nt, q0.begin() + (size_t)(m + 1) * nt, k.primInf[m]);
    *out = ctx;
    return phx_set_state(ctx, PHX_Q, q0.data(), (int64_t)q0.size());
}

int phx_ctx_destroy(phx_ctx *ctx)
{
    if (!ctx) return PHX_OK;
    cudaStreamSynchronize(ctx->stream);
    if (ctx->aux) {
        cudaStreamSynchronize(ctx->aux);
        cudaStreamDestroy(ctx->aux);
        cudaEventDestroy(ctx->evFork);
        cudaEventDestroy(ctx->evHead);
    }
    for (void *p : ctx->allocs) cudaFree(p);
    delete ctx;
    return PHX_OK;
}

const char *phx_last_error(const phx_ctx *ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int phx_set_stream(phx_ctx *ctx, void *stream)
{
    if (!ctx) return PHX_ERR_ARG;
    ctx->stream = (cudaStream_t)stream;
    return PHX_OK;
}

int phx_device(const phx_ctx *ctx) { return ctx ? ctx->device : -1; }
int phx_set_step(phx_ctx *ctx, int step) { if (!ctx || step < 0) return PHX_ERR_ARG; ctx->step = step; return PHX_OK; }
int phx_get_step(const phx_ctx *ctx) { return ctx ? ctx->step : -1; }
int64_t phx_launch_count(const phx_ctx *ctx) { return ctx ? ctx->launches : -1; }

// --- state I/O -------------------------------------------------------------
}  // extern "C"

namespace {

int check_launch(phx_ctx *ctx, int n = 1)
{
    ctx->launches += n;
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(ctx, PHX_ERR_CUDA, std::string("kernel launch failed: ") + cudaGetErrorString(e));
    return PHX_OK;
}

template <class T> const TurbWork<T> &turb_of(const phx_ctx *ctx);
template <> const TurbWork<double> &turb_of<double>(const phx_ctx *ctx) { return ctx->t64; }
template <> const TurbWork<float> &turb_of<float>(const phx_ctx *ctx) { return ctx->t32; }

// Fills ctx->tmp with the selected array in the reference's order; returns the
// number of rows and the row length (elements per row).
template <class T>
int export_work(phx_ctx *ctx, const Work<T> &w, int which, int &rows, int &len)
{
    const DevGrid &g = ctx->g;
    const int nt = ctx->nTotal, nc = ctx->nCell;
    cudaStream_t s = ctx->stream;
    PHX_CUDA(ctx, cudaMemsetAsync(ctx->tmp, 0, sizeof(double) * 5 * (size_t)nt, s));
    switch (which) {
    case PHX_RES: rows = 5; len = nt; launch_export<T>(g, w.crec, kC, 0, 5, 1, nc, ctx->tmp, nt, s); break;
    case PHX_LIMIT:   // first order with a limiter: zero on the ghosts too (ComputeLimiter :18215)
        rows = 1; len = nt;
        launch_export<T>(g, w.qrec, kQ, 7, 1, 1, ctx->nc.firstOrder && ctx->nc.limiter != PHX_LIMITER_NOLIM ? nc : nt,
                         ctx->tmp, nt, s);
        break;
    case PHX_GRADX: rows = 5; len = nt; launch_export<T>(g, w.grec, kG, 0, 5, 3, nc, ctx->tmp, nt, s); break;
    case PHX_GRADY: rows = 5; len = nt; launch_export<T>(g, w.grec, kG, 1, 5, 3, nc, ctx->tmp, nt, s); break;
    case PHX_GRADZ: rows = 5; len = nt; launch_export<T>(g, w.grec, kG, 2, 5, 3, nc, ctx->tmp, nt, s); break;
    case PHX_DQ: rows = 5; len = nt; launch_export<T>(g, w.dqrec, kD, 0, 5, 1, nt, ctx->tmp, nt, s); break;
    case PHX_INVSPEC: rows = 1; len = nc; launch_export<T>(g, w.crec, kC, 6, 1, 1, nc, ctx->tmp, nc, s); break;
    case PHX_VISSPEC: rows = 1; len = nc; launch_export<T>(g, w.crec, kC, 7, 1, 1, nc, ctx->tmp, nc, s); break;
    case PHX_DT: rows = 1; len = nt; launch_export<T>(g, w.dtraw, 1, 0, 1, 1, nc, ctx->tmp, nt, s); break;
    case PHX_SA_SRC:
        if (!ctx->sa || !ctx->nc.saSource) return fail(ctx, PHX_ERR_ARG, "PHX_SA_SRC needs the learned SA source");
        rows = 1; len = nc;
        launch_export<T>(g, turb_of<T>(ctx).tsrc, 1, 0, 1, 1, nc, ctx->tmp, nc, s);
        break;
    case PHX_GRAD_TURB:
        if (!ctx->sa) return fail(ctx, PHX_ERR_ARG, "PHX_GRAD_TURB needs the SA model");
        rows = 3; len = nt;
        launch_export<T>(g, turb_of<T>(ctx).tgrad, kTg, 0, 3, 1, nc, ctx->tmp, nt, s);
        break;
    case PHX_Q_TURB:
    case PHX_VISL:
    case PHX_VIST:
    case PHX_RES_TURB: {
        if (!ctx->sa) return fail(ctx, PHX_ERR_ARG, "SA state selector on a context without the SA model");
        const TurbWork<T> &t = turb_of<T>(ctx);
        rows = 1; len = nt;
        if (which == PHX_Q_TURB) launch_export<double>(g, t.qt64, 1, 0, 1, 1, nt, ctx->tmp, nt, s);
        else if (which == PHX_VISL) launch_export<T>(g, w.trec, kTr, 2, 1, 1, nt, ctx->tmp, nt, s);
        else if (which == PHX_VIST) launch_export<T>(g, w.trec, kTr, 1, 1, 1, nt, ctx->tmp, nt, s);
        else launch_export<T>(g, t.tcrec, kTc, 0, 1, 1, nc, ctx->tmp, nt, s);
        break;
    }
    default: return fail(ctx, PHX_ERR_ARG, "unknown or unavailable state selector");
    }
    return check_launch(ctx, 2);
}

}  // namespace

extern "C" {

static int get_state_impl(phx_ctx *ctx, int which, double *dst, int64_t n, bool hostSide)
{
    if (!ctx || !dst) return PHX_ERR_ARG;
    const int nt = ctx->nTotal, nc = ctx->nCell;
    int rows = 0, len = 0, rc;
    if (which == PHX_Q) {
        rows = 5; len = nt;
        launch_export_q(ctx->g, ctx->q64[ctx->cur], ctx->tmp, ctx->stream);
        rc = check_launch(ctx);
    } else {
        rc = ctx->mixed ? export_work(ctx, ctx->w32, which, rows, len) : export_work(ctx, ctx->w64, which, rows, len);
    }
    if (rc) return rc;
    if (n != (int64_t)rows * len) return fail(ctx, PHX_ERR_ARG, "state size does not match the selector");
    if (which == PHX_DT) {
        // the reference's dt after ReduceMaxTimeStep (NSSolverUnstruct.cpp:5717-5745):
        // min(dt, ktmax min dt) / vol, ghosts copied from their owners
        std::vector<double> raw(nt);
        Reduce red;
        PHX_CUDA(ctx, cudaMemcpyAsync(raw.data(), ctx->tmp, sizeof(double) * nt, cudaMemcpyDeviceToHost, ctx->stream));
        PHX_CUDA(ctx, cudaMemcpyAsync(&red, ctx->red, sizeof(Reduce), cudaMemcpyDeviceToHost, ctx->stream));
        PHX_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        double mindt;
        std::memcpy(&mindt, &red.mindt_bits, sizeof(double));
        for (int c = 0; c < nc; ++c) {
            double d = raw[c];
            if (ctx->nc.ktmax > 0) d = std::min(d, ctx->nc.ktmax * mindt);
            raw[c] = d / ctx->geom[10][c];
        }
        for (int f = 0; f < ctx->nBFace; ++f) raw[nc + f] = 0.0;
        // ghost dt: the owner's value (SetGhostCell)
        std::vector<int2> lr(ctx->nBFace);
        std::vector<int> orig(ctx->nTotal);
        if (ctx->nBFace) {
            PHX_CUDA(ctx, cudaMemcpy(lr.data(), ctx->g.lr, sizeof(int2) * ctx->nBFace, cudaMemcpyDeviceToHost));
            PHX_CUDA(ctx, cudaMemcpy(orig.data(), ctx->g.orig, sizeof(int) * ctx->nTotal, cudaMemcpyDeviceToHost));
            for (int fs = 0; fs < ctx->nBFace; ++fs) raw[orig[nc + fs]] = raw[orig[lr[fs].x]];
        }
        if (hostSide) std::memcpy(dst, raw.data(), sizeof(double) * nt);
        else PHX_CUDA(ctx, cudaMemcpy(dst, raw.data(), sizeof(double) * nt, cudaMemcpyHostToDevice));
        return PHX_OK;
    }
    PHX_CUDA(ctx, cudaMemcpyAsync(dst, ctx->tmp, sizeof(double) * n, hostSide ? cudaMemcpyDeviceToHost
                                                                             : cudaMemcpyDeviceToDevice, ctx->stream));
    PHX_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return PHX_OK;
}

static int set_state_impl(phx_ctx *ctx, int which, const double *src, int64_t n, bool hostSide)
{
    if (!ctx || !src) return PHX_ERR_ARG;
    const int nt = ctx->nTotal;
    if (which == PHX_VIST) {
        if (!ctx->sa) return fail(ctx, PHX_ERR_ARG, "SA state selector on a context without the SA model");
        if (n != (int64_t)nt) return fail(ctx, PHX_ERR_ARG, "state size does not match the selector");
        PHX_CUDA(ctx, cudaMemcpyAsync(ctx->tmp, src, sizeof(double) * n, hostSide ? cudaMemcpyHostToDevice
                                                                                 : cudaMemcpyDeviceToDevice, ctx->stream));
        if (ctx->mixed) launch_import_vist<float>(ctx->g, ctx->tmp, ctx->w32, ctx->stream);
        else launch_import_vist<double>(ctx->g, ctx->tmp, ctx->w64, ctx->stream);
        int rc = check_launch(ctx);
        if (rc) return rc;
        PHX_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        return PHX_OK;
    }
    if (which == PHX_Q_TURB) {
        if (!ctx->sa) return fail(ctx, PHX_ERR_ARG, "SA state selector on a context without the SA model");
        if (n != (int64_t)nt) return fail(ctx, PHX_ERR_ARG, "state size does not match the selector");
        PHX_CUDA(ctx, cudaMemcpyAsync(ctx->tmp, src, sizeof(double) * n, hostSide ? cudaMemcpyHostToDevice
                                                                                 : cudaMemcpyDeviceToDevice, ctx->stream));
        if (ctx->mixed) launch_import_turb<float>(ctx->g, ctx->tmp, ctx->t32, ctx->w32, ctx->stream);
        else launch_import_turb<double>(ctx->g, ctx->tmp, ctx->t64, ctx->w64, ctx->stream);
        ctx->turbNodeValid = false;   // GG-node: a loaded nu~ forms its node values afresh
        int rc = check_launch(ctx);
        if (rc) return rc;
        PHX_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        return PHX_OK;
    }
    if (which != PHX_Q) return fail(ctx, PHX_ERR_ARG, "only PHX_Q, PHX_Q_TURB and PHX_VIST can be set");
    if (n != (int64_t)5 * nt) return fail(ctx, PHX_ERR_ARG, "state size does not match the selector");
    PHX_CUDA(ctx, cudaMemcpyAsync(ctx->tmp, src, sizeof(double) * n, hostSide ? cudaMemcpyHostToDevice
                                                                             : cudaMemcpyDeviceToDevice, ctx->stream));
    launch_import_q(ctx->g, ctx->tmp, ctx->q64[ctx->cur], ctx->stream);
    if (ctx->mixed) launch_sync_qrec<float>(ctx->g, ctx->nc, ctx->q64[ctx->cur], ctx->w32, ctx->stream);
    else launch_sync_qrec<double>(ctx->g, ctx->nc, ctx->q64[ctx->cur], ctx->w64, ctx->stream);
    ctx->nodePrev = false;   // GG-node: a loaded state starts its node values afresh, as a restart does
    int rc = check_launch(ctx, 2);
    if (rc) return rc;
    PHX_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return PHX_OK;
}

int phx_set_state(phx_ctx *ctx, int which, const double *host, int64_t n) { return set_state_impl(ctx, which, host, n, true); }
int phx_get_state(phx_ctx *ctx, int which, double *host, int64_t n) { return get_state_impl(ctx, which, host, n, true); }
int phx_set_state_device(phx_ctx *ctx, int which, const double *dev, int64_t n) { return set_state_impl(ctx, which, dev, n, false); }
int phx_get_state_device(phx_ctx *ctx, int which, double *dev, int64_t n) { return get_state_impl(ctx, which, dev, n, false); }

int phx_get_geometry(phx_ctx *ctx, const char *name, double *host, int64_t n)
{
    if (!ctx || !name || !host) return PHX_ERR_ARG;
    for (int i = 0; i < 12; ++i) {
        if (std::strcmp(name, kGeomNames[i]) == 0) {
            if ((size_t)n != ctx->geom[i].size()) return fail(ctx, PHX_ERR_ARG, "geometry size mismatch");
            std::memcpy(host, ctx->geom[i].data(), sizeof(double) * n);
            return PHX_OK;
        }
    }
    return fail(ctx, PHX_ERR_ARG, std::string("unknown geometry array ") + name);
}

// --- phases ----------------------------------------------------------------

static double cfl_at(const NsConst &c, int step)
{
    // NSSolver::ComputeCFL, CFD/NSSolver/src/NSSolver.cpp:595-668 (cflMethod 0)
    if (step >= c.cflVaryStep) return c.cflEnd;
    return c.cflStart + (c.cflEnd - c.cflStart) * step / c.cflVaryStep;
}

int phx_ns_boundary(phx_ctx *ctx)
{
    if (!ctx) return PHX_ERR_ARG;
    if (ctx->mixed) launch_boundary<float>(ctx->g, ctx->nc, ctx->q64[ctx->cur], ctx->w32, ctx->stream);
    else launch_boundary<double>(ctx->g, ctx->nc, ctx->q64[ctx->cur], ctx->w64, ctx->stream);
    return check_launch(ctx);
}

// Flow initialisation (Simulation::PreSolve, Main/src/Simulation.cpp:1190-1237):
// isInIniting holds for outer steps 1..flowInitStep.  Then the limiter is zero
// (NSSolverUnstruct::ComputeLimiter, :18203-18224), the face states are the
// cell values (ReConstructFaceValue, :14014-14021) and the inviscid flux is Van
// Leer's (ComputeInviscidFlux, :14229-14235).
static void init_phase(phx_ctx *ctx)
{
    const bool init = ctx->prm.flowInitStep > 0 && ctx->step <= ctx->prm.flowInitStep;
    // the "1st" limiter is first order at every step, with the configured scheme
    ctx->nc.firstOrder = init || ctx->prm.uns_limiter_name == PHX_LIMITER_FIRST ? 1 : 0;
    ctx->nc.scheme = init ? PHX_SCHEME_VANLEER : ctx->prm.uns_scheme_name;
}

int phx_ns_gradient_limiter(phx_ctx *ctx)
{
    if (!ctx) return PHX_ERR_ARG;
    init_phase(ctx);
    const int prev = ctx->nodePrev ? 1 : 0;
    if (ctx->mixed) launch_gradient_limiter<float>(ctx->g, ctx->nc, ctx->w32, prev, ctx->stream);
    else launch_gradient_limiter<double>(ctx->g, ctx->nc, ctx->w64, prev, ctx->stream);
    ctx->nodePrev = true;
    return check_launch(ctx);
}

int phx_ns_residual(phx_ctx *ctx)
{
    if (!ctx) return PHX_ERR_ARG;
    init_phase(ctx);
    launch_reset_reduce(ctx->red, ctx->stream);
    const double cfl = cfl_at(ctx->nc, ctx->step);
    if (ctx->mixed) launch_residual<float>(ctx->g, ctx->nc, ctx->w32, ctx->red, cfl, ctx->stream);
    else launch_residual<double>(ctx->g, ctx->nc, ctx->w64, ctx->red, cfl, ctx->stream);
    ctx->haveResidual = true;
    return check_launch(ctx, 3);
}

static int ns_lusgs(phx_ctx *ctx, int sweeps)
{
    if (!ctx->haveResidual) return fail(ctx, PHX_ERR_STATE, "the LU-SGS sweeps need phx_ns_residual first");
    if (sweeps == kSweepBackward && !ctx->nsForwardDone)
        return fail(ctx, PHX_ERR_STATE, "phx_ns_lusgs_backward needs phx_ns_lusgs_forward first");
    const int e = ctx->mixed
                      ? launch_lusgs<float>(ctx->g, ctx->nc, ctx->w32, ctx->red, ctx->numSMs, ctx->stream, sweeps)
                      : launch_lusgs<double>(ctx->g, ctx->nc, ctx->w64, ctx->red, ctx->numSMs, ctx->stream, sweeps);
    if (e) return fail(ctx, PHX_ERR_CUDA, std::string("cooperative launch failed: ") + cudaGetErrorString((cudaError_t)e));
    ctx->nsForwardDone = sweeps == kSweepForward;
    return check_launch(ctx, (sweeps & kSweepForward) ? 2 : 1);
}

static int refuse_zone(phx_ctx *ctx, const char *what)
{
    return fail(ctx, PHX_ERR_STATE, std::string(what) +
                                        ": the grid has interface faces; run the phases with the halo exchanges "
                                        "(phx_ns_lusgs_forward / phx_ns_lusgs_backward and the SA pair)");
}

int phx_ns_lusgs(phx_ctx *ctx)
{
    if (!ctx) return PHX_ERR_ARG;
    if (ctx->hasInterface) return refuse_zone(ctx, "phx_ns_lusgs");
    return ns_lusgs(ctx, kSweepBoth);
}

int phx_ns_lusgs_forward(phx_ctx *ctx) { return ctx ? ns_lusgs(ctx, kSweepForward) : PHX_ERR_ARG; }
int phx_ns_lusgs_backward(phx_ctx *ctx) { return ctx ? ns_lusgs(ctx, kSweepBackward) : PHX_ERR_ARG; }

int phx_ns_update(phx_ctx *ctx)
{
    if (!ctx) return PHX_ERR_ARG;
    const int nxt = 1 - ctx->cur;
    double *qo = ctx->q64[ctx->cur], *qn = ctx->q64[nxt];
    if (ctx->mixed) {
        launch_update<float>(ctx->g, ctx->nc, ctx->w32, qo, qn, ctx->red, ctx->neglist, ctx->numSMs, ctx->stream);
        launch_solution_fix<float>(ctx->g, ctx->nc, ctx->w32, qo, qn, ctx->red, ctx->neglist, ctx->stream);
    } else {
        launch_update<double>(ctx->g, ctx->nc, ctx->w64, qo, qn, ctx->red, ctx->neglist, ctx->numSMs, ctx->stream);
        launch_solution_fix<double>(ctx->g, ctx->nc, ctx->w64, qo, qn, ctx->red, ctx->neglist, ctx->stream);
    }
    ctx->cur = nxt;
    // Controller::PostSolve (Controller.cpp:5063-5090): ghost states of the
    // updated field (the SA step and exported states read them)
    if (ctx->mixed) launch_boundary_post<float>(ctx->g, ctx->nc, ctx->q64[ctx->cur], ctx->w32, ctx->stream);
    else launch_boundary_post<double>(ctx->g, ctx->nc, ctx->q64[ctx->cur], ctx->w64, ctx->stream);
    return check_launch(ctx, 3);
}

int phx_sa_boundary(phx_ctx *ctx)
{
    if (!ctx) return PHX_ERR_ARG;
    if (!ctx->sa) return fail(ctx, PHX_ERR_STATE, "the context has no SA model (viscousType != 3)");
    if (ctx->mixed) launch_sa_boundary<float>(ctx->g, ctx->nc, ctx->q64[ctx->cur], ctx->w32, ctx->t32, ctx->stream);
    else launch_sa_boundary<double>(ctx->g, ctx->nc, ctx->q64[ctx->cur], ctx->w64, ctx->t64, ctx->stream);
    return check_launch(ctx);
}

int phx_sa_residual(phx_ctx *ctx)
{
    if (!ctx) return PHX_ERR_ARG;
    if (!ctx->sa) return fail(ctx, PHX_ERR_STATE, "the context has no SA model (viscousType != 3)");
    if (!ctx->haveResidual) return fail(ctx, PHX_ERR_STATE, "phx_sa_residual needs the NS time step (phx_ns_residual)");
    if (ctx->nc.saSource && !ctx->mlpReady)
        return fail(ctx, PHX_ERR_STATE, "sa_source selects the learned source but no model is set (phx_mlp_train / phx_mlp_set)");
    const MlpDev *mlp = ctx->nc.saSource ? &ctx->mlp : nullptr;
    if (ctx->prm.gradientName == 2 && !ctx->turbNodeValid) {
        // GG-node: the nu~ node values of the state as initialised or loaded, before any boundary
        if (ctx->mixed) launch_turb_node_values<float>(ctx->g, ctx->w32, ctx->t32, ctx->stream);
        else launch_turb_node_values<double>(ctx->g, ctx->w64, ctx->t64, ctx->stream);
        ctx->turbNodeValid = true;
    }
    if (ctx->mixed)
        launch_sa_residual<float>(ctx->g, ctx->nc, ctx->q64[ctx->cur], ctx->w32, ctx->t32, ctx->red, mlp, ctx->nmlp,
                                  ctx->numSMs, ctx->stream);
    else
        launch_sa_residual<double>(ctx->g, ctx->nc, ctx->q64[ctx->cur], ctx->w64, ctx->t64, ctx->red, mlp, ctx->nmlp,
                                   ctx->numSMs, ctx->stream);
    return check_launch(ctx, mlp ? 6 : 5);
}

static int sa_lusgs(phx_ctx *ctx, int sweeps)
{
    if (!ctx->sa) return fail(ctx, PHX_ERR_STATE, "the context has no SA model (viscousType != 3)");
    if (sweeps == kSweepBackward && !ctx->saForwardDone)
        return fail(ctx, PHX_ERR_STATE, "phx_sa_lusgs_backward needs phx_sa_lusgs_forward first");
    const int e = ctx->mixed ? launch_sa_lusgs<float>(ctx->g, ctx->nc, ctx->w32, ctx->t32, ctx->red, ctx->numSMs,
                                                      ctx->stream, sweeps)
                             : launch_sa_lusgs<double>(ctx->g, ctx->nc, ctx->w64, ctx->t64, ctx->red, ctx->numSMs,
                                                       ctx->stream, sweeps);
    if (e) return fail(ctx, PHX_ERR_CUDA, std::string("cooperative launch failed: ") + cudaGetErrorString((cudaError_t)e));
    ctx->saForwardDone = sweeps == kSweepForward;
    return check_launch(ctx, (sweeps & kSweepForward) ? 2 : 1);
}

int phx_sa_lusgs(phx_ctx *ctx)
{
    if (!ctx) return PHX_ERR_ARG;
    if (ctx->hasInterface) return refuse_zone(ctx, "phx_sa_lusgs");
    return sa_lusgs(ctx, kSweepBoth);
}

int phx_sa_lusgs_forward(phx_ctx *ctx) { return ctx ? sa_lusgs(ctx, kSweepForward) : PHX_ERR_ARG; }
int phx_sa_lusgs_backward(phx_ctx *ctx) { return ctx ? sa_lusgs(ctx, kSweepBackward) : PHX_ERR_ARG; }

int phx_sa_update(phx_ctx *ctx)
{
    if (!ctx) return PHX_ERR_ARG;
    if (!ctx->sa) return fail(ctx, PHX_ERR_STATE, "the context has no SA model (viscousType != 3)");
    if (ctx->mixed) launch_sa_update<float>(ctx->g, ctx->nc, ctx->w32, ctx->t32, ctx->stream);
    else launch_sa_update<double>(ctx->g, ctx->nc, ctx->w64, ctx->t64, ctx->stream);
    int rc = check_launch(ctx);
    if (rc) return rc;
    rc = phx_sa_boundary(ctx);   // TURB PostSolve
    if (rc || ctx->prm.gradientName != 2) return rc;
    // GG-node: PostSolve forms the nu~ node values the next SA gradient reads
    // (Controller::PostSolve, Controller.cpp:5063-5205)
    if (ctx->mixed) launch_turb_node_values<float>(ctx->g, ctx->w32, ctx->t32, ctx->stream);
    else launch_turb_node_values<double>(ctx->g, ctx->w64, ctx->t64, ctx->stream);
    ctx->turbNodeValid = true;
    return check_launch(ctx);
}

// One outer step.  With `headDone` the step's NS boundary, gradient and
// residual have already run on the second stream (see below) and are only
// joined, before the NS sweep.  With `prefetch` and SA, the next step's NS
// boundary, gradient and residual are issued on the second stream right after
// this step's SA residual, so that they run while the latency-bound SA sweep
// and SA update run.  They need the updated NS state and the eddy viscosity,
// which the SA residual has formed (the SA update changes nu~ only, and the SA
// boundary after it writes the ghosts' eddy viscosity again with the same
// values); they write ghost states, gradients, the limiter, the laminar
// viscosity slot, the face fluxes and LU-SGS factors, the NS residual record,
// the time step and the NS reduction fields, none of which the SA sweep, SA
// update or SA boundary reads (they read the SA records, the owner cells'
// FP64 state and the eddy viscosity).  The two cooperative sweeps never
// overlap: the NS sweep waits for both streams.
static int relax_one(phx_ctx *ctx, double *dhist, int i, bool headDone, bool prefetch, bool &prefetched)
{
    ctx->step += 1;   // Simulation::UpdateOuterIterationStep
    prefetched = false;
    int rc;
    if (headDone) {
        PHX_CUDA(ctx, cudaStreamWaitEvent(ctx->stream, ctx->evHead, 0));
    } else {
        if ((rc = phx_ns_boundary(ctx))) return rc;
        if ((rc = phx_ns_gradient_limiter(ctx))) return rc;
        if ((rc = phx_ns_residual(ctx))) return rc;
    }
    if ((rc = phx_ns_lusgs(ctx))) return rc;
    if ((rc = phx_ns_update(ctx))) return rc;
    launch_finish_step(ctx->red, dhist, i, (double)ctx->nCell, ctx->stream);
    if (ctx->sa) {
        if ((rc = phx_sa_residual(ctx))) return rc;
        if (prefetch) {
            PHX_CUDA(ctx, cudaEventRecord(ctx->evFork, ctx->stream));
            PHX_CUDA(ctx, cudaStreamWaitEvent(ctx->aux, ctx->evFork, 0));
            cudaStream_t main = ctx->stream;
            ctx->stream = ctx->aux;
            ctx->step += 1;   // the next step's flow-initialisation phase and CFL
            rc = phx_ns_boundary(ctx);
            if (!rc) rc = phx_ns_gradient_limiter(ctx);
            if (!rc) rc = phx_ns_residual(ctx);
            ctx->step -= 1;
            ctx->stream = main;
            if (rc) return rc;
            PHX_CUDA(ctx, cudaEventRecord(ctx->evHead, ctx->aux));
            prefetched = true;
        }
        if ((rc = phx_sa_lusgs(ctx))) return rc;
        if ((rc = phx_sa_update(ctx))) return rc;
    }
    return check_launch(ctx);
}

int phx_ns_relaxation(phx_ctx *ctx, int nsteps, double *res_hist)
{
    if (!ctx || nsteps < 0) return PHX_ERR_ARG;
    if (ctx->hasInterface) return refuse_zone(ctx, "phx_ns_relaxation");
    if (nsteps > ctx->histCap) {
        double *h = nullptr;
        const int rc = dalloc(ctx, &h, (size_t)nsteps);
        if (rc) return rc;
        ctx->hist = h;
        ctx->histCap = nsteps;
    }
    // the overlap of the SA tail with the next step's NS head (relax_one);
    // PHX_OVERLAP=0 runs every phase on the context's stream, in order
    const char *ov = getenv("PHX_OVERLAP");
    const bool overlap = ctx->sa && !(ov && atoi(ov) == 0);
    if (overlap && !ctx->aux) {
        PHX_CUDA(ctx, cudaStreamCreateWithFlags(&ctx->aux, cudaStreamNonBlocking));
        PHX_CUDA(ctx, cudaEventCreateWithFlags(&ctx->evFork, cudaEventDisableTiming));
        PHX_CUDA(ctx, cudaEventCreateWithFlags(&ctx->evHead, cudaEventDisableTiming));
    }
    bool headDone = false;
    for (int i = 0; i < nsteps; ++i) {
        bool prefetched = false;
        const int rc = relax_one(ctx, ctx->hist, i, headDone, overlap && i + 1 < nsteps, prefetched);
        if (rc) {
            // nothing of this call stays in flight on the second stream
            if (prefetched) cudaStreamWaitEvent(ctx->stream, ctx->evHead, 0);
            return rc;
        }
        headDone = prefetched;
    }
    Reduce red;
    PHX_CUDA(ctx, cudaMemcpyAsync(&red, ctx->red, sizeof(Reduce), cudaMemcpyDeviceToHost, ctx->stream));
    if (res_hist && nsteps > 0)
        PHX_CUDA(ctx, cudaMemcpyAsync(res_hist, ctx->hist, sizeof(double) * nsteps, cudaMemcpyDeviceToHost, ctx->stream));
    PHX_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (red.error != 0) {
        // reported once: the next call starts with a clear status
        PHX_CUDA(ctx, cudaMemsetAsync(&ctx->red->error, 0, sizeof(int), ctx->stream));
        PHX_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    }
    if (red.error == PHX_ERR_TIMEOUT) return fail(ctx, PHX_ERR_TIMEOUT, "LU-SGS dependency wait timed out");
    if (red.error == PHX_ERR_NUMERIC) return fail(ctx, PHX_ERR_NUMERIC, "residual is not finite (divergence)");
    return PHX_OK;
}

// ---------------------------------------------------------------------------
// Partitioned grids: SwapGeometry, the halo plan and its exchanges, the
// minimum time step over all zones.
// ---------------------------------------------------------------------------
int phx_swap_geometry(phx_ctx *ctx, int64_t n, const int32_t *bfaces, const double *xcc, const double *ycc,
                      const double *zcc, const double *vol, double avg_vol)
{
    if (!ctx || n < 0 || (n > 0 && (!bfaces || !xcc || !ycc || !zcc || !vol))) return PHX_ERR_ARG;
    if (!ctx->hasInterface) return fail(ctx, PHX_ERR_STATE, "the grid has no interface faces");
    const int nc = ctx->nCell, nb = ctx->nBFace, nf = ctx->nFace, nt = ctx->nTotal;
    for (int64_t i = 0; i < n; ++i)
        if (bfaces[i] < 0 || bfaces[i] >= nb || !ctx->itfFace[bfaces[i]])
            return fail(ctx, PHX_ERR_ARG, "phx_swap_geometry: not an interface face");
    PHX_CUDA(ctx, cudaStreamSynchronize(ctx->stream));   // the records below may be in use
    for (int64_t i = 0; i < n; ++i) {
        const int re = nc + bfaces[i];
        ctx->geom[7][re] = xcc[i];
        ctx->geom[8][re] = ycc[i];
        ctx->geom[9][re] = zcc[i];
        ctx->geom[10][re] = vol[i];
    }
    HostGrid h{};
    h.nCell = nc; h.nBFace = nb; h.nFace = nf; h.nNode = ctx->nNode;
    h.left = ctx->hleft;
    h.right = ctx->hright;
    const phx_params *prm = &ctx->prm;
    // face records (least-squares weight in slot 7), ghost centres, cell matrices
    std::vector<double> iwt, m6;
    if (prm->gradientName == 1) lsq_weights(h, ctx->geom, iwt, m6);
    std::vector<double> frec((size_t)nf * kF), xrec((size_t)nt * kX);
    for (int fs = 0; fs < nf; ++fs) {
        const int f = ctx->forder[fs];
        for (int k = 0; k < 7; ++k) frec[(size_t)fs * kF + k] = ctx->geom[k][f];
        frec[(size_t)fs * kF + 7] = prm->gradientName == 1 ? iwt[f] : 0.0;
    }
    for (int i = 0; i < nt; ++i) {
        const int c = i < nc ? ctx->ord[i] : nc + ctx->forder[i - nc];
        for (int k = 0; k < 4; ++k) xrec[(size_t)i * kX + k] = ctx->geom[7 + k][c];
    }
    PHX_CUDA(ctx, cudaMemcpy(const_cast<double *>(ctx->g.frec), frec.data(), sizeof(double) * frec.size(),
                             cudaMemcpyHostToDevice));
    PHX_CUDA(ctx, cudaMemcpy(const_cast<double *>(ctx->g.xrec), xrec.data(), sizeof(double) * xrec.size(),
                             cudaMemcpyHostToDevice));
    if (prm->gradientName == 1) {
        std::vector<double> lsqs((size_t)nc * 8, 0.0);
        for (int i = 0; i < nc; ++i)
            for (int k = 0; k < 6; ++k) lsqs[(size_t)i * 8 + k] = m6[(size_t)ctx->ord[i] * 6 + k];
        PHX_CUDA(ctx, cudaMemcpy(const_cast<double *>(ctx->g.lsq), lsqs.data(), sizeof(double) * lsqs.size(),
                                 cudaMemcpyHostToDevice));
    }
    if (prm->viscousType) {
        const std::vector<uint8_t> vref = viscous_flags(h, ctx->geom, prm->skewnessAngle, prm->turbSkewnessAngle);
        std::vector<uint8_t> vflag(nf);
        for (int fs = 0; fs < nf; ++fs) vflag[fs] = vref[ctx->forder[fs]];
        PHX_CUDA(ctx, cudaMemcpy(const_cast<uint8_t *>(ctx->g.vflag), vflag.data(), nf, cudaMemcpyHostToDevice));
    }
    if (avg_vol > 0.0) {
        // the Venkatakrishnan threshold scales with the average cell volume of all zones
        const double K = prm->venkatCoeff;
        double kt = K * K * K;
        kt *= 1.0 / std::pow(std::pow(avg_vol, 1.0 / 3.0), 3.0);
        ctx->nc.venkatK3 = kt;
        ctx->g.avgVol = avg_vol;
    }
    return PHX_OK;
}

int phx_set_halo(phx_ctx *ctx, int64_t n_send, const int32_t *send_cells, int64_t n_recv, const int32_t *recv_bfaces)
{
    if (!ctx || n_send < 0 || n_recv < 0 || (n_send > 0 && !send_cells) || (n_recv > 0 && !recv_bfaces))
        return PHX_ERR_ARG;
    if (!ctx->hasInterface) return fail(ctx, PHX_ERR_STATE, "the grid has no interface faces");
    // a cell may be sent more than once (one row per interface face behind
    // it, to one or several zones), so only the receive side is bounded by a
    // grid count: every interface face is received once
    if (n_send > INT32_MAX || n_recv > ctx->nBFace) return PHX_ERR_ARG;
    std::vector<int> snd((size_t)n_send), rcv((size_t)n_recv);
    for (int64_t i = 0; i < n_send; ++i) {
        if (send_cells[i] < 0 || send_cells[i] >= ctx->nCell) return fail(ctx, PHX_ERR_ARG, "phx_set_halo: bad cell");
        snd[i] = ctx->rankOf[send_cells[i]];
    }
    for (int64_t i = 0; i < n_recv; ++i) {
        const int f = recv_bfaces[i];
        if (f < 0 || f >= ctx->nBFace || !ctx->itfFace[f])
            return fail(ctx, PHX_ERR_ARG, "phx_set_halo: not an interface face");
        rcv[i] = ctx->nCell + ctx->bfacePos[f];
    }
    int rc = 0;
    const int *ds = nullptr, *dr = nullptr;
    if (n_send > 0) rc |= upload(ctx, &ds, snd);
    if (n_recv > 0) rc |= upload(ctx, &dr, rcv);
    if (rc) return rc < 0 ? rc : PHX_ERR_CUDA;
    ctx->haloSend = const_cast<int *>(ds);
    ctx->haloRecv = const_cast<int *>(dr);
    ctx->nHaloSend = (int)n_send;
    ctx->nHaloRecv = (int)n_recv;
    return PHX_OK;
}

static bool halo_field_ok(const phx_ctx *ctx, int field)
{
    if (field == PHX_HALO_TURB) return ctx->sa;
    return field >= PHX_HALO_Q && field <= PHX_HALO_DQ;
}

int64_t phx_halo_row_bytes(const phx_ctx *ctx, int field)
{
    if (!ctx || !halo_field_ok(ctx, field)) return PHX_ERR_ARG;
    return (int64_t)(ctx->mixed ? halo_row_bytes<float>(field) : halo_row_bytes<double>(field));
}

int phx_halo_pack(phx_ctx *ctx, int field, void *buf_dev)
{
    if (!ctx || !halo_field_ok(ctx, field) || (ctx->nHaloSend > 0 && !buf_dev)) return PHX_ERR_ARG;
    if (!ctx->hasInterface) return fail(ctx, PHX_ERR_STATE, "the grid has no interface faces");
    unsigned char *b = static_cast<unsigned char *>(buf_dev);
    if (ctx->mixed)
        launch_halo_pack<float>(ctx->g, field, ctx->q64[ctx->cur], ctx->w32, ctx->t32, ctx->haloSend, ctx->nHaloSend,
                                b, ctx->stream);
    else
        launch_halo_pack<double>(ctx->g, field, ctx->q64[ctx->cur], ctx->w64, ctx->t64, ctx->haloSend,
                                 ctx->nHaloSend, b, ctx->stream);
    return check_launch(ctx, ctx->nHaloSend > 0 ? 1 : 0);
}

int phx_halo_unpack(phx_ctx *ctx, int field, const void *buf_dev)
{
    if (!ctx || !halo_field_ok(ctx, field) || (ctx->nHaloRecv > 0 && !buf_dev)) return PHX_ERR_ARG;
    if (!ctx->hasInterface) return fail(ctx, PHX_ERR_STATE, "the grid has no interface faces");
    const unsigned char *b = static_cast<const unsigned char *>(buf_dev);
    if (ctx->mixed)
        launch_halo_unpack<float>(ctx->g, ctx->nc, field, ctx->q64[ctx->cur], ctx->w32, ctx->t32, ctx->haloRecv,
                                  ctx->nHaloRecv, b, ctx->stream);
    else
        launch_halo_unpack<double>(ctx->g, ctx->nc, field, ctx->q64[ctx->cur], ctx->w64, ctx->t64, ctx->haloRecv,
                                   ctx->nHaloRecv, b, ctx->stream);
    return check_launch(ctx, ctx->nHaloRecv > 0 ? 1 : 0);
}

int phx_ns_min_timestep(phx_ctx *ctx, double *out)
{
    if (!ctx || !out) return PHX_ERR_ARG;
    if (!ctx->haveResidual) return fail(ctx, PHX_ERR_STATE, "phx_ns_min_timestep needs phx_ns_residual first");
    unsigned long long bits = 0;
    PHX_CUDA(ctx, cudaMemcpyAsync(&bits, &ctx->red->mindt_bits, sizeof(bits), cudaMemcpyDeviceToHost, ctx->stream));
    PHX_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    double v;
    std::memcpy(&v, &bits, sizeof(v));
    *out = v;
    return PHX_OK;
}

int phx_ns_set_min_timestep(phx_ctx *ctx, double value)
{
    if (!ctx || !(value > 0.0)) return PHX_ERR_ARG;
    unsigned long long bits;
    std::memcpy(&bits, &value, sizeof(bits));
    PHX_CUDA(ctx, cudaMemcpyAsync(&ctx->red->mindt_bits, &bits, sizeof(bits), cudaMemcpyHostToDevice, ctx->stream));
    PHX_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return PHX_OK;
}

int phx_step_status(phx_ctx *ctx)
{
    if (!ctx) return PHX_ERR_ARG;
    int err = 0;
    PHX_CUDA(ctx, cudaMemcpyAsync(&err, &ctx->red->error, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    PHX_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (err != 0) {
        PHX_CUDA(ctx, cudaMemsetAsync(&ctx->red->error, 0, sizeof(int), ctx->stream));
        PHX_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    }
    if (err == PHX_ERR_TIMEOUT) return fail(ctx, PHX_ERR_TIMEOUT, "LU-SGS dependency wait timed out");
    if (err == PHX_ERR_NUMERIC) return fail(ctx, PHX_ERR_NUMERIC, "residual is not finite (divergence)");
    return PHX_OK;
}

// ---------------------------------------------------------------------------
// Restart files: the content of the reference's restart (Version, outnstep,
// nTotalCell, q; with SA q_turb and visturb) and the learned-source model.
// Layout (little-endian): "PHXRST01", int32 version, int32 flags (1: SA
// arrays, 2: model), int64 nCell, nBFace, outnstep, then q [5][nTotal], with
// SA q_turb [nTotal] and visturb [nTotal] (FP64, reference order), and with a
// model int64 n and n floats.
// ---------------------------------------------------------------------------
static const char kRestartMagic[8] = {'P', 'H', 'X', 'R', 'S', 'T', '0', '1'};
static constexpr int32_t kRestartVersion = 1;

int phx_write_restart(phx_ctx *ctx, const char *path)
{
    if (!ctx || !path) return PHX_ERR_ARG;
    const int64_t nt = ctx->nTotal;
    std::vector<double> q((size_t)(5 * nt)), qt, vt;
    int rc = phx_get_state(ctx, PHX_Q, q.data(), 5 * nt);
    if (rc) return rc;
    if (ctx->sa) {
        qt.resize((size_t)nt);
        vt.resize((size_t)nt);
        if ((rc = phx_get_state(ctx, PHX_Q_TURB, qt.data(), nt))) return rc;
        if ((rc = phx_get_state(ctx, PHX_VIST, vt.data(), nt))) return rc;
    }
    const bool model = ctx->sa && ctx->mlpReady;
    FILE *f = fopen(path, "wb");
    if (!f) return fail(ctx, PHX_ERR_ARG, std::string("cannot write ") + path);
    const int32_t hdr[2] = {kRestartVersion, (ctx->sa ? 1 : 0) | (model ? 2 : 0)};
    const int64_t sizes[3] = {ctx->nCell, ctx->nBFace, ctx->step};
    bool ok = fwrite(kRestartMagic, 1, 8, f) == 8 && fwrite(hdr, sizeof(hdr), 1, f) == 1 &&
              fwrite(sizes, sizeof(sizes), 1, f) == 1 && fwrite(q.data(), sizeof(double), q.size(), f) == q.size();
    if (ok && ctx->sa)
        ok = fwrite(qt.data(), sizeof(double), qt.size(), f) == qt.size() &&
             fwrite(vt.data(), sizeof(double), vt.size(), f) == vt.size();
    if (ok && model) {
        const int64_t n = (int64_t)ctx->mlpBlob.size();
        ok = fwrite(&n, sizeof(n), 1, f) == 1 && fwrite(ctx->mlpBlob.data(), sizeof(float), (size_t)n, f) == (size_t)n;
    }
    ok = (fclose(f) == 0) && ok;
    return ok ? PHX_OK : fail(ctx, PHX_ERR_ARG, std::string("short write to ") + path);
}

int phx_read_restart(phx_ctx *ctx, const char *path)
{
    if (!ctx || !path) return PHX_ERR_ARG;
    FILE *f = fopen(path, "rb");
    if (!f) return fail(ctx, PHX_ERR_ARG, std::string("cannot read ") + path);
    char magic[8];
    int32_t hdr[2];
    int64_t sizes[3];
    auto bad = [&](const char *why) {
        fclose(f);
        return fail(ctx, PHX_ERR_ARG, std::string("restart ") + path + ": " + why);
    };
    if (fread(magic, 1, 8, f) != 8 || std::memcmp(magic, kRestartMagic, 8) != 0) return bad("not a phx restart file");
    if (fread(hdr, sizeof(hdr), 1, f) != 1 || hdr[0] != kRestartVersion) return bad("unknown version");
    if (fread(sizes, sizeof(sizes), 1, f) != 1) return bad("short header");
    // as TurbSolverUnstr::ReadRestartH5 checks nTotalCell against the grid (TurbSolverUnstr.cpp:669-676)
    if (sizes[0] != ctx->nCell || sizes[1] != ctx->nBFace) return bad("cell or boundary-face count differs from the grid");
    if (((hdr[1] & 1) != 0) != ctx->sa) return bad("SA arrays present in one of file and context only");
    if (sizes[2] < 0 || sizes[2] > 0x7fffffff) return bad("bad step");
    const int64_t nt = ctx->nTotal;
    std::vector<double> q((size_t)(5 * nt)), qt, vt;
    if (fread(q.data(), sizeof(double), q.size(), f) != q.size()) return bad("short q");
    if (ctx->sa) {
        qt.resize((size_t)nt);
        vt.resize((size_t)nt);
        if (fread(qt.data(), sizeof(double), qt.size(), f) != qt.size() ||
            fread(vt.data(), sizeof(double), vt.size(), f) != vt.size())
            return bad("short SA arrays");
    }
    std::vector<float> blob;
    if (hdr[1] & 2) {
        int64_t n = 0;
        if (fread(&n, sizeof(n), 1, f) != 1 || n != kMlpBlobFloats) return bad("bad model size");
        blob.resize((size_t)n);
        if (fread(blob.data(), sizeof(float), blob.size(), f) != blob.size()) return bad("short model");
    }
    fclose(f);
    int rc = phx_set_state(ctx, PHX_Q, q.data(), 5 * nt);
    if (!rc && ctx->sa) rc = phx_set_state(ctx, PHX_Q_TURB, qt.data(), nt);
    if (!rc && ctx->sa) rc = phx_set_state(ctx, PHX_VIST, vt.data(), nt);
    if (!rc && !blob.empty()) rc = phx_mlp_set(ctx, blob.data(), (int64_t)blob.size());
    if (!rc) ctx->step = (int)sizes[2];   // outnstep: the CFL ramp and the flow-initialisation phase resume
    return rc;
}

int phx_set_wait_limit(phx_ctx *ctx, int64_t polls)
{
    if (!ctx) return PHX_ERR_ARG;
    if (polls <= 0) return fail(ctx, PHX_ERR_ARG, "the wait limit must be positive");
    ctx->nc.spinLimit = polls;
    return PHX_OK;
}

int phx_fault_hold_cell(phx_ctx *ctx, int32_t cell)
{
    if (!ctx) return PHX_ERR_ARG;
    if (cell < -1 || cell >= ctx->nCell) return fail(ctx, PHX_ERR_ARG, "cell out of range");
    ctx->nc.holdCell = cell < 0 ? -1 : ctx->rankOf[cell];
    return PHX_OK;
}

// --- learned SA source ----------------------------------------------------

static int mlp_install(phx_ctx *ctx, const float *blob)
{
    MlpHostWeights w;
    std::memcpy(&w, blob, sizeof(MlpHostWeights));
    const float *norm = blob + kMlpWeightFloats;
    std::vector<uint16_t> w1c, w2c, w3c;
    mlp_pack(w, w1c, w2c, w3c);
    std::vector<uint16_t> wall(w1c);
    wall.insert(wall.end(), w2c.begin(), w2c.end());
    wall.insert(wall.end(), w3c.begin(), w3c.end());
    std::vector<float> fall;
    fall.insert(fall.end(), w.b1, w.b1 + kMlpH);
    fall.insert(fall.end(), w.b2, w.b2 + kMlpH);
    fall.insert(fall.end(), w.b3, w.b3 + kMlpH);
    fall.insert(fall.end(), w.w4, w.w4 + kMlpH);
    PHX_CUDA(ctx, cudaMemcpy(ctx->mlpW, wall.data(), sizeof(uint16_t) * wall.size(), cudaMemcpyHostToDevice));
    PHX_CUDA(ctx, cudaMemcpy(ctx->mlpF, fall.data(), sizeof(float) * fall.size(), cudaMemcpyHostToDevice));
    MlpDev &m = ctx->mlp;
    m.w1c = ctx->mlpW;
    m.w2c = ctx->mlpW + kMlpH * kMlpK1;
    m.w3c = ctx->mlpW + kMlpH * kMlpK1 + kMlpH * kMlpH;
    m.b1 = ctx->mlpF;
    m.b2 = ctx->mlpF + kMlpH;
    m.b3 = ctx->mlpF + 2 * kMlpH;
    m.w4 = ctx->mlpF + 3 * kMlpH;
    m.b4 = w.b4;
    for (int k = 0; k < kMlpIn; ++k) {
        m.mean[k] = norm[k];
        m.rstd[k] = norm[kMlpIn + k];
        m.lo[k] = norm[2 * kMlpIn + k];
        m.hi[k] = norm[3 * kMlpIn + k];
    }
    m.tscale = norm[4 * kMlpIn];
    std::vector<uint8_t> occ(kMlpGrid * kMlpGrid);
    for (int b = 0; b < kMlpGrid * kMlpGrid; ++b) occ[b] = norm[4 * kMlpIn + 1 + b] != 0.0f ? 1 : 0;
    PHX_CUDA(ctx, cudaMemcpy(ctx->mlpOcc, occ.data(), occ.size(), cudaMemcpyHostToDevice));
    m.occ = ctx->mlpOcc;
    ctx->mlpBlob.assign(blob, blob + kMlpBlobFloats);
    ctx->mlpReady = true;
    return PHX_OK;
}

int phx_sa_capture(phx_ctx *ctx, float *features, float *targets, int32_t *cells, float *scales, int64_t capacity,
                   int64_t *count)
{
    if (!ctx || !features || !targets || !count || capacity < 0) return PHX_ERR_ARG;
    if (!ctx->sa) return fail(ctx, PHX_ERR_STATE, "the context has no SA model (viscousType != 3)");
    if (!ctx->haveResidual) return fail(ctx, PHX_ERR_STATE, "phx_sa_capture needs a completed SA residual");
    const int nc = ctx->nCell;
    float *df = nullptr, *dt = nullptr, *dsc = nullptr;
    int *dcl = nullptr;
    unsigned long long *dn = nullptr;
    int rc = 0;
    rc |= dalloc(ctx, &df, (size_t)nc * kMlpIn);
    rc |= dalloc(ctx, &dt, (size_t)nc);
    rc |= dalloc(ctx, &dsc, (size_t)nc);
    rc |= dalloc(ctx, &dcl, (size_t)nc);
    rc |= dalloc(ctx, &dn, 1);
    if (rc) return rc;
    PHX_CUDA(ctx, cudaMemsetAsync(dn, 0, sizeof(unsigned long long), ctx->stream));
    if (ctx->mixed) launch_mlp_capture<float>(ctx->g, ctx->nc, ctx->w32, ctx->t32, df, dt, dcl, dsc, nc, dn, ctx->stream);
    else launch_mlp_capture<double>(ctx->g, ctx->nc, ctx->w64, ctx->t64, df, dt, dcl, dsc, nc, dn, ctx->stream);
    rc = check_launch(ctx);
    if (rc) return rc;
    unsigned long long n = 0;
    PHX_CUDA(ctx, cudaMemcpyAsync(&n, dn, sizeof(n), cudaMemcpyDeviceToHost, ctx->stream));
    PHX_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    const int64_t m = std::min<int64_t>((int64_t)n, capacity);
    PHX_CUDA(ctx, cudaMemcpy(features, df, sizeof(float) * kMlpIn * (size_t)m, cudaMemcpyDeviceToHost));
    PHX_CUDA(ctx, cudaMemcpy(targets, dt, sizeof(float) * (size_t)m, cudaMemcpyDeviceToHost));
    if (cells) PHX_CUDA(ctx, cudaMemcpy(cells, dcl, sizeof(int) * (size_t)m, cudaMemcpyDeviceToHost));
    if (scales) PHX_CUDA(ctx, cudaMemcpy(scales, dsc, sizeof(float) * (size_t)m, cudaMemcpyDeviceToHost));
    // the staging buffers are released at once (they are not part of the context's resident state)
    for (void *p : {(void *)df, (void *)dt, (void *)dsc, (void *)dcl, (void *)dn}) {
        ctx->allocs.erase(std::find(ctx->allocs.begin(), ctx->allocs.end(), p));
        cudaFree(p);
    }
    *count = m;
    return PHX_OK;
}

int phx_mlp_train(phx_ctx *ctx, const float *features, const float *targets, int64_t n, int epochs, int batch,
                  double lr, uint64_t seed, double *final_loss)
{
    if (!ctx || !features || !targets || n < 2 || epochs < 1 || batch < 1 || !(lr > 0.0)) return PHX_ERR_ARG;
    std::vector<float> blob(kMlpBlobFloats);
    MlpHostWeights w;
    float *norm = blob.data() + kMlpWeightFloats;
    float tscale = 1.0f;
    double loss = 0.0;
    const int e = mlp_train(features, targets, n, epochs, batch, (float)lr, seed, w, norm, norm + kMlpIn,
                            norm + 2 * kMlpIn, norm + 3 * kMlpIn, norm + 4 * kMlpIn + 1, tscale, loss, ctx->stream);
    if (e) return fail(ctx, PHX_ERR_CUDA, std::string("MLP training failed: ") + cudaGetErrorString((cudaError_t)e));
    norm[4 * kMlpIn] = tscale;
    std::memcpy(blob.data(), &w, sizeof(MlpHostWeights));
    if (final_loss) *final_loss = loss;
    return mlp_install(ctx, blob.data());
}

int phx_mlp_get(phx_ctx *ctx, float *blob, int64_t n)
{
    if (!ctx || !blob) return PHX_ERR_ARG;
    if (!ctx->mlpReady) return fail(ctx, PHX_ERR_STATE, "no learned source model is set");
    if (n != kMlpBlobFloats) return fail(ctx, PHX_ERR_ARG, "model blob size mismatch");
    std::memcpy(blob, ctx->mlpBlob.data(), sizeof(float) * kMlpBlobFloats);
    return PHX_OK;
}

int phx_mlp_set(phx_ctx *ctx, const float *blob, int64_t n)
{
    if (!ctx || !blob) return PHX_ERR_ARG;
    if (!ctx->sa) return fail(ctx, PHX_ERR_STATE, "the context has no SA model (viscousType != 3)");
    if (n != kMlpBlobFloats) return fail(ctx, PHX_ERR_ARG, "model blob size mismatch");
    return mlp_install(ctx, blob);
}

int64_t phx_mlp_blob_size(void) { return kMlpBlobFloats; }

int64_t phx_mlp_param_count(void) { return mlp_param_count(); }

int phx_mlp_loss_grad(const float *params, int64_t nparam, const float *x, const float *y, int64_t n, float *grad,
                      double *loss)
{
    if (!params || !x || !y || !grad || !loss || nparam != mlp_param_count() || n < 1 || n > (1 << 24))
        return PHX_ERR_ARG;
    double l = 0.0;
    const int e = mlp_loss_grad(params, x, y, (int)n, grad, l, nullptr);
    if (e) return PHX_ERR_CUDA;
    *loss = l;
    return PHX_OK;
}

int phx_mlp_cells(phx_ctx *ctx, uint64_t *count)
{
    if (!ctx || !count) return PHX_ERR_ARG;
    if (!ctx->sa) return fail(ctx, PHX_ERR_STATE, "the context has no SA model (viscousType != 3)");
    unsigned long long n = 0;
    PHX_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    PHX_CUDA(ctx, cudaMemcpy(&n, ctx->nmlp, sizeof(n), cudaMemcpyDeviceToHost));
    *count = n;
    return PHX_OK;
}

int phx_forces(phx_ctx *ctx, double out[16])
{
    if (!ctx || !out) return PHX_ERR_ARG;
    if (ctx->mixed) launch_forces<float>(ctx->g, ctx->nc, ctx->w32, ctx->q64[ctx->cur], ctx->forces, ctx->stream);
    else launch_forces<double>(ctx->g, ctx->nc, ctx->w64, ctx->q64[ctx->cur], ctx->forces, ctx->stream);
    int rc = check_launch(ctx);
    if (rc) return rc;
    PHX_CUDA(ctx, cudaMemcpyAsync(out, ctx->forces, sizeof(double) * 16, cudaMemcpyDeviceToHost, ctx->stream));
    PHX_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return PHX_OK;
}

int phx_residual_norm(phx_ctx *ctx, double out[5])
{
    if (!ctx || !out) return PHX_ERR_ARG;
    double *d = ctx->forces;   // 16-double device scratch of the context, free between calls
    if (ctx->mixed) launch_resnorm<float>(ctx->g, ctx->w32, d, ctx->numSMs, ctx->stream);
    else launch_resnorm<double>(ctx->g, ctx->w64, d, ctx->numSMs, ctx->stream);
    const int rc = check_launch(ctx);
    if (rc) return rc;
    double s[5];
    PHX_CUDA(ctx, cudaMemcpyAsync(s, d, sizeof(double) * 5, cudaMemcpyDeviceToHost, ctx->stream));
    PHX_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    for (int m = 0; m < 5; ++m) out[m] = std::sqrt(s[m] / ctx->nCell);
    return PHX_OK;
}

}  // extern "C"
