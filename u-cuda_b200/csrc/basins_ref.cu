// Basins of attraction, reference method (run_basins, parametric_engine.cpp:6035-6510):
// classes and features per cell (ucb_basins_ref.cuh, NVRTC), then the DBSCAN of the
// features.
//
// The reference clusters with a host loop: per cluster it launches a seed search over all
// cells, then one kernel over all cells per member to find that member's unlabelled
// neighbours within eps (minPts = 1), so a map of N cells costs about N launches of N
// threads. Its result is fixed by three rules: fixed-point seeds first (lowest index,
// cluster ids -1, -2, ...), then oscillating seeds (lowest index, ids 1, 2, ...); a
// cluster is everything reachable from its seed through cells within eps of each other;
// unbound cells are never expanded and end unlabelled. That is: clusters are the connected
// components of the "distance <= eps" graph over the classified cells, numbered by the
// lowest fixed-point index they contain (negative ids) or else by their lowest
// oscillating index (positive ids). Here the components come from a grid in feature
// space: cells are binned into squares of side 0.7 eps (two cells of one square are
// within eps of each other, so a square is connected by construction), squares are sorted,
// neighbouring squares up to two apart are joined (atomic union-find) when any pair of
// their cells is within eps, and the components are ranked by their lowest fixed-point /
// oscillating cell with a radix sort.
#include <cuda_runtime.h>

#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <string>
#include <vector>

#include "csv_export.h"
#include "engine_internal.h"

namespace ucbbr {

constexpr long long kExcluded = 0x7FFFFFFFFFFFFFFFLL;   // unbound cells (last square)
constexpr long long kSingleton = 0x7FFFFFFFFFFFFFFELL;  // cells that join nothing: own square
constexpr double kMaxSquare = 2305843009213693952.0;     // 2^61 squares from the origin
constexpr unsigned int kNone = 0xFFFFFFFFu;
constexpr int kPairInline = 1024;  // pair products searched by the square's own thread

// Feature bounding box of a square as order-preserving integer keys (dkey).
struct Box {
    long long x0, x1, y0, y1;
};

__device__ __forceinline__ unsigned long long ordered(long long v) {
    return (unsigned long long)v ^ 0x8000000000000000ULL;
}

// Order-preserving map of a double to a signed integer (for atomicMin / atomicMax); it is
// its own inverse.
__device__ __forceinline__ long long dkey(double v) {
    const long long b = __double_as_longlong(v);
    return b >= 0 ? b : (b ^ 0x7FFFFFFFFFFFFFFFLL);
}
__device__ __forceinline__ double dval(long long k) {
    return __longlong_as_double(k >= 0 ? k : (k ^ 0x7FFFFFFFFFFFFFFFLL));
}

// Grid square of every cell, and the first sort's keys (y) and values (cell index).
// Cells with non-finite features are at distance NaN / inf from every cell, so in the
// reference they join nothing and form clusters of their own; cells more than 2^61
// squares from the origin (features beyond ~1.6e18 eps) are treated the same way.
// Single precision: the features are first rounded to float, the numb the reference
// clusters in (so that the geometry below and the distance test see the same values).
__global__ void bin_kernel(double* f1, double* f2, const int* cls, long long n, double side, int single,
                           long long* bx, long long* by, unsigned long long* key, unsigned int* idx) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double v1 = f1[i], v2 = f2[i];
    if (single) {
        v1 = (double)(float)v1;
        v2 = (double)(float)v2;
        f1[i] = v1;
        f2[i] = v2;
    }
    long long x, y;
    const double qx = floor(v1 / side), qy = floor(v2 / side);
    if (cls[i] == 0) {
        x = kExcluded;
        y = kExcluded;
    } else if (!(fabs(qx) <= kMaxSquare) || !(fabs(qy) <= kMaxSquare)) {
        x = kSingleton;
        y = i;
    } else {
        x = (long long)qx;
        y = (long long)qy;
    }
    bx[i] = x;
    by[i] = y;
    key[i] = ordered(y);
    idx[i] = (unsigned int)i;
}

__global__ void gather_key_kernel(const long long* bx, const unsigned int* order, long long n,
                                  unsigned long long* key) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    key[i] = ordered(bx[order[i]]);
}

// In (x, y)-sorted order: square boundaries, and the features gathered contiguously.
__global__ void head_kernel(const long long* bx, const long long* by, const unsigned int* order, const double* f1,
                            const double* f2, long long n, unsigned int* head, double* sf1, double* sf2) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const unsigned int a = order[i];
    sf1[i] = f1[a];
    sf2[i] = f2[a];
    if (i == 0) {
        head[i] = 1;
        return;
    }
    const unsigned int b = order[i - 1];
    head[i] = (bx[a] != bx[b] || by[a] != by[b]) ? 1u : 0u;
}

// sq_of holds the inclusive scan of the square heads; the square of cell i is one less.
__global__ void squares_kernel(const long long* bx, const long long* by, const unsigned int* order,
                               const unsigned int* head, unsigned int* sq_of, long long n, unsigned int* start,
                               long long* sx, long long* sy) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const unsigned int s = sq_of[i] - 1u;
    sq_of[i] = s;
    if (!head[i]) return;
    start[s] = (unsigned int)i;
    sx[s] = bx[order[i]];
    sy[s] = by[order[i]];
}

__global__ void init_squares_kernel(unsigned int nsq, long long n, unsigned int* start, unsigned int* parent,
                                    Box* box, unsigned int* min_fp, unsigned int* min_osc, int* comp_label) {
    const unsigned int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s > nsq) return;
    if (s == nsq) {
        start[s] = (unsigned int)n;  // sentinel: end of the last square
        return;
    }
    parent[s] = s;
    box[s] = Box{kExcluded, -kExcluded, kExcluded, -kExcluded};
    min_fp[s] = kNone;
    min_osc[s] = kNone;
    comp_label[s] = 0;
}

// Bounding box of every square's features and its lowest fixed-point / oscillating cell.
// Cells are in square order, so a warp mostly covers one square: reduce across the warp
// then, and fall back to one atomic per lane at square boundaries.
__global__ void square_stats_kernel(const double* sf1, const double* sf2, const unsigned int* order,
                                    const unsigned int* sq_of, const int* cls, const long long* sx, long long n,
                                    Box* box, unsigned int* min_fp, unsigned int* min_osc) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const bool live = i < n;
    const unsigned int s = live ? sq_of[i] : kNone;
    const bool boxed = live && sx[s] != kExcluded && sx[s] != kSingleton;
    const unsigned int c = live ? order[i] : kNone;
    const int k = live ? cls[c] : 0;
    long long x0 = boxed ? dkey(sf1[i]) : kExcluded, x1 = boxed ? dkey(sf1[i]) : -kExcluded;
    long long y0 = boxed ? dkey(sf2[i]) : kExcluded, y1 = boxed ? dkey(sf2[i]) : -kExcluded;
    unsigned int fp = k == -1 ? c : kNone, osc = k == 1 ? c : kNone;
    const unsigned int s0 = __shfl_sync(0xFFFFFFFFu, s, 0);
    if (__all_sync(0xFFFFFFFFu, s == s0)) {
        for (int o = 16; o > 0; o >>= 1) {
            x0 = min(x0, __shfl_xor_sync(0xFFFFFFFFu, x0, o));
            x1 = max(x1, __shfl_xor_sync(0xFFFFFFFFu, x1, o));
            y0 = min(y0, __shfl_xor_sync(0xFFFFFFFFu, y0, o));
            y1 = max(y1, __shfl_xor_sync(0xFFFFFFFFu, y1, o));
        }
        fp = __reduce_min_sync(0xFFFFFFFFu, fp);
        osc = __reduce_min_sync(0xFFFFFFFFu, osc);
        if ((threadIdx.x & 31) != 0 || s == kNone) return;
    }
    if (!live) return;
    if (x0 != kExcluded) {
        atomicMin(&box[s].x0, x0);
        atomicMax(&box[s].x1, x1);
        atomicMin(&box[s].y0, y0);
        atomicMax(&box[s].y1, y1);
    }
    if (fp != kNone) atomicMin(&min_fp[s], fp);
    if (osc != kNone) atomicMin(&min_osc[s], osc);
}

// Parent links are changed by atomics (in L2) from any SM, so they are read past L1
// (__ldcg): a stale link could make a CAS below fail forever. Links only ever point to a
// smaller square index, so the walk ends within nsq steps.
__device__ __forceinline__ unsigned int find_root(unsigned int* parent, unsigned int v) {
    unsigned int p = __ldcg(&parent[v]);
    while (p != v) {
        const unsigned int g = __ldcg(&parent[p]);
        if (g != p) atomicCAS(&parent[v], p, g);  // path halving
        v = p;
        p = __ldcg(&parent[v]);
    }
    return v;
}

// Lock-free union: the larger root is linked under the smaller one.
__device__ __forceinline__ void unite(unsigned int* parent, unsigned int a, unsigned int b) {
    for (;;) {
        a = find_root(parent, a);
        b = find_root(parent, b);
        if (a == b) return;
        if (a > b) {
            const unsigned int t = a;
            a = b;
            b = t;
        }
        if (atomicCAS(&parent[b], b, a) == b) return;
    }
}

// The reference's neighbour test, sqrt(dx^2 + dy^2) <= eps, in numb (float when single),
// rounded operation by operation (no contraction into FMA).
__device__ __forceinline__ bool within(double ax, double ay, double bx, double by, double eps, int single) {
    if (single) {
        const float dx = __fsub_rn((float)ax, (float)bx), dy = __fsub_rn((float)ay, (float)by);
        return sqrtf(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy))) <= (float)eps;
    }
    const double dx = __dsub_rn(ax, bx), dy = __dsub_rn(ay, by);
    return sqrt(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy))) <= eps;
}

// Every square is joined with the squares up to two steps ahead of it (the other half of
// its 5 x 5 neighbourhood joins it from the other side): skipped when the boxes are
// surely more than eps apart, joined outright when every pair is surely within eps,
// otherwise searched pair by pair — here for small squares, by a whole CTA later
// (heavy list) for large ones. The margins cover the rounding of the reference's test
// (a few ulp of numb).
__global__ void join_kernel(const double* sf1, const double* sf2, const unsigned int* start, const long long* sx,
                            const long long* sy, const Box* box, unsigned int nsq, double eps, int single,
                            unsigned int* parent, uint2* heavy, unsigned int* n_heavy) {
    const unsigned int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nsq || sx[s] == kExcluded || sx[s] == kSingleton) return;
    const double margin = single ? 1e-5 : 1e-9;
    const double lo2 = eps * eps * (1.0 - margin), hi2 = eps * eps * (1.0 + margin);
    const unsigned int a0 = start[s], a1 = start[s + 1];
    const Box ka = box[s];
    const double ax0 = dval(ka.x0), ax1 = dval(ka.x1), ay0 = dval(ka.y0), ay1 = dval(ka.y1);
    for (int dx = 0; dx <= 2; ++dx) {
        for (int dy = -2; dy <= 2; ++dy) {
            if (dx == 0 && dy <= 0) continue;
            const long long tx = sx[s] + dx, ty = sy[s] + dy;
            unsigned int lo = 0, hi = nsq;  // binary search of (tx, ty) among the sorted squares
            while (lo < hi) {
                const unsigned int mid = (lo + hi) >> 1;
                if (sx[mid] < tx || (sx[mid] == tx && sy[mid] < ty)) lo = mid + 1;
                else hi = mid;
            }
            if (lo >= nsq || sx[lo] != tx || sy[lo] != ty) continue;
            const unsigned int t = lo;
            const Box kb = box[t];
            const double bx0 = dval(kb.x0), bx1 = dval(kb.x1), by0 = dval(kb.y0), by1 = dval(kb.y1);
            const double gx = fmax(0.0, fmax(bx0 - ax1, ax0 - bx1)), gy = fmax(0.0, fmax(by0 - ay1, ay0 - by1));
            if (gx * gx + gy * gy > hi2) continue;
            const double fx = fmax(ax1, bx1) - fmin(ax0, bx0), fy = fmax(ay1, by1) - fmin(ay0, by0);
            if (fx * fx + fy * fy < lo2) {
                unite(parent, s, t);
                continue;
            }
            if (find_root(parent, s) == find_root(parent, t)) continue;
            const unsigned int b0 = start[t], b1 = start[t + 1];
            if ((unsigned long long)(a1 - a0) * (b1 - b0) > (unsigned long long)kPairInline) {
                heavy[atomicAdd(n_heavy, 1u)] = make_uint2(s, t);
                continue;
            }
            bool hit = false;
            for (unsigned int i = a0; i < a1 && !hit; ++i)
                for (unsigned int j = b0; j < b1 && !hit; ++j) hit = within(sf1[i], sf2[i], sf1[j], sf2[j], eps, single);
            if (hit) unite(parent, s, t);
        }
    }
}

// Pair search of the heavy square pairs: one CTA per pair, threads striding over the
// first square's cells, stopping as soon as any thread finds a pair within eps.
__global__ void __launch_bounds__(256) heavy_join_kernel(const double* sf1, const double* sf2,
                                                         const unsigned int* start, const uint2* heavy,
                                                         const unsigned int* n_heavy, double eps, int single,
                                                         unsigned int* parent) {
    __shared__ int found;
    const unsigned int count = *n_heavy;
    for (unsigned int w = blockIdx.x; w < count; w += gridDim.x) {
        const unsigned int s = heavy[w].x, t = heavy[w].y;
        if (threadIdx.x == 0) found = find_root(parent, s) == find_root(parent, t) ? 1 : 0;
        __syncthreads();
        const unsigned int a0 = start[s], a1 = start[s + 1], b0 = start[t], b1 = start[t + 1];
        for (unsigned int i = a0 + threadIdx.x; i < a1; i += blockDim.x) {
            if (*(volatile int*)&found) break;
            const double x = sf1[i], y = sf2[i];
            for (unsigned int j = b0; j < b1; ++j) {
                if (within(x, y, sf1[j], sf2[j], eps, single)) {
                    found = 2;
                    break;
                }
                if (((j - b0) & 63) == 63 && *(volatile int*)&found) break;
            }
        }
        __syncthreads();
        if (threadIdx.x == 0 && found == 2) unite(parent, s, t);
        __syncthreads();
    }
}

// Components (root squares): lowest fixed-point and oscillating cell of each.
__global__ void root_stats_kernel(unsigned int* parent, const unsigned int* min_fp, const unsigned int* min_osc,
                                  unsigned int nsq, unsigned int* root_fp, unsigned int* root_osc) {
    const unsigned int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nsq) return;
    const unsigned int r = find_root(parent, s);
    parent[s] = r;
    if (min_fp[s] != kNone) atomicMin(&root_fp[r], min_fp[s]);
    if (min_osc[s] != kNone) atomicMin(&root_osc[r], min_osc[s]);
}

// Sort keys of the components: fixed-point components by their lowest fixed point, the
// others by their lowest oscillating cell; kNone (sorted last) for non-roots.
__global__ void rank_keys_kernel(const unsigned int* parent, const unsigned int* root_fp, const unsigned int* root_osc,
                                 unsigned int nsq, unsigned int* kfp, unsigned int* kosc, unsigned int* ids) {
    const unsigned int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nsq) return;
    const bool root = parent[s] == s;
    kfp[s] = root ? root_fp[s] : kNone;
    kosc[s] = (root && root_fp[s] == kNone) ? root_osc[s] : kNone;
    ids[s] = s;
}

__global__ void assign_rank_kernel(const unsigned int* keys, const unsigned int* roots, unsigned int nsq, int sign,
                                   int* comp_label) {
    const unsigned int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nsq || keys[i] == kNone) return;
    comp_label[roots[i]] = sign * (int)(i + 1);
}

__global__ void label_kernel(const unsigned int* order, const unsigned int* sq_of, const unsigned int* parent,
                             const long long* sx, const int* comp_label, long long n, int* labels) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const unsigned int s = sq_of[i];
    labels[order[i]] = sx[s] == kExcluded ? 0 : comp_label[parent[s]];
}

}  // namespace ucbbr

namespace ucb {
namespace {

constexpr int kMaxAmountOfX = 32;
constexpr int kMaxAmountOfValues = 64;

// Stream-ordered device allocations of one call, released (and the stream drained) when
// the call returns.
struct DeviceArena {
    ucb_engine* e;
    cudaStream_t st;
    std::vector<void*> ptrs;
    std::string err;
    ~DeviceArena() {
        for (void* p : ptrs) cudaFreeAsync(p, st);
        cudaStreamSynchronize(st);
    }
    template <class T>
    T* get(size_t count) {
        void* p = nullptr;
        const cudaError_t ce = dev_alloc(e, &p, std::max<size_t>(count, 1) * sizeof(T), st);
        if (ce != cudaSuccess) {
            err = std::string("cudaMallocAsync: ") + cudaGetErrorString(ce);
            return nullptr;
        }
        ptrs.push_back(p);
        return static_cast<T*>(p);
    }
};

struct EventPair {
    cudaEvent_t a = nullptr, b = nullptr;
    EventPair() {
        cudaEventCreate(&a);
        cudaEventCreate(&b);
    }
    ~EventPair() {
        cudaEventDestroy(a);
        cudaEventDestroy(b);
    }
};

template <class R>
int fail(ucb_engine* e, R* r, int code, const std::string& msg) {
    e->last_error = msg;
    std::snprintf(r->error, sizeof r->error, "%s", msg.c_str());
    r->ok = 0;
    return code;
}

// Clusters n cells: features f1 / f2 (device, rewritten as float values when single) and
// classes cls into labels lab. Enqueues everything on st; reads back the square count
// once (4 bytes). Returns the number of its own kernel launches, or -1 with err set.
int cluster_features(ucb_engine* e, cudaStream_t st, DeviceArena& mem, double* d_f1, double* d_f2, const int* d_cls,
                     unsigned int N, double eps, int single, int* d_lab, std::string& err) {
    long long* bx = mem.get<long long>(N);
    long long* by = mem.get<long long>(N);
    unsigned long long* k_in = mem.get<unsigned long long>(N);
    unsigned long long* k_out = mem.get<unsigned long long>(N);
    unsigned int* v_in = mem.get<unsigned int>(N);
    unsigned int* order = mem.get<unsigned int>(N);
    unsigned int* head = mem.get<unsigned int>(N);
    unsigned int* sq_of = mem.get<unsigned int>(N);
    double* sf1 = mem.get<double>(N);
    double* sf2 = mem.get<double>(N);
    unsigned int* counts = mem.get<unsigned int>(4);  // [2]: heavy square pairs
    if (!bx || !by || !k_in || !k_out || !v_in || !order || !head || !sq_of || !sf1 || !sf2 || !counts) {
        err = mem.err;
        return -1;
    }
    const unsigned int B = 256, G = (N + B - 1) / B;
    ucbbr::bin_kernel<<<G, B, 0, st>>>(d_f1, d_f2, d_cls, N, 0.7 * eps, single, bx, by, k_in, v_in);
    size_t sort_bytes = 0, scan_bytes = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, k_in, k_out, v_in, order, (int)N, 0, 64, st);
    cub::DeviceScan::InclusiveSum(nullptr, scan_bytes, head, sq_of, (int)N, st);
    const size_t tmp_bytes = std::max(sort_bytes, scan_bytes);
    void* tmp = mem.get<char>(tmp_bytes);
    if (!tmp) {
        err = mem.err;
        return -1;
    }
    // stable LSD order: by y, then by x
    cub::DeviceRadixSort::SortPairs(tmp, sort_bytes, k_in, k_out, v_in, order, (int)N, 0, 64, st);
    ucbbr::gather_key_kernel<<<G, B, 0, st>>>(bx, order, N, k_in);
    cudaMemcpyAsync(v_in, order, (size_t)N * 4, cudaMemcpyDeviceToDevice, st);
    cub::DeviceRadixSort::SortPairs(tmp, sort_bytes, k_in, k_out, v_in, order, (int)N, 0, 64, st);
    ucbbr::head_kernel<<<G, B, 0, st>>>(bx, by, order, d_f1, d_f2, N, head, sf1, sf2);
    cub::DeviceScan::InclusiveSum(tmp, scan_bytes, head, sq_of, (int)N, st);
    unsigned int nsq = 0;  // squares: the last inclusive-scan entry
    cudaMemcpyAsync(&nsq, sq_of + (N - 1), 4, cudaMemcpyDeviceToHost, st);
    cudaError_t ce = cudaStreamSynchronize(st);
    if (ce != cudaSuccess) {
        err = std::string("CUDA basins clustering: ") + cudaGetErrorString(ce);
        return -1;
    }
    unsigned int* start = mem.get<unsigned int>((size_t)nsq + 1);
    long long* sx = mem.get<long long>(nsq);
    long long* sy = mem.get<long long>(nsq);
    ucbbr::Box* box = mem.get<ucbbr::Box>(nsq);
    unsigned int* parent = mem.get<unsigned int>(nsq);
    unsigned int* min_fp = mem.get<unsigned int>(nsq);
    unsigned int* min_osc = mem.get<unsigned int>(nsq);
    unsigned int* root_fp = mem.get<unsigned int>(nsq);
    unsigned int* root_osc = mem.get<unsigned int>(nsq);
    int* comp_label = mem.get<int>(nsq);
    uint2* heavy = mem.get<uint2>((size_t)nsq * 12);
    if (!start || !sx || !sy || !box || !parent || !min_fp || !min_osc || !root_fp || !root_osc || !comp_label ||
        !heavy) {
        err = mem.err;
        return -1;
    }
    const unsigned int GS = (nsq + B) / B;  // nsq + 1 threads
    ucbbr::init_squares_kernel<<<GS, B, 0, st>>>(nsq, N, start, parent, box, min_fp, min_osc, comp_label);
    ucbbr::squares_kernel<<<G, B, 0, st>>>(bx, by, order, head, sq_of, N, start, sx, sy);
    ucbbr::square_stats_kernel<<<G, B, 0, st>>>(sf1, sf2, order, sq_of, d_cls, sx, N, box, min_fp, min_osc);
    cudaMemsetAsync(counts + 2, 0, 4, st);
    ucbbr::join_kernel<<<GS, B, 0, st>>>(sf1, sf2, start, sx, sy, box, nsq, eps, single, parent, heavy, counts + 2);
    ucbbr::heavy_join_kernel<<<e->sm_count * 4, 256, 0, st>>>(sf1, sf2, start, heavy, counts + 2, eps, single,
                                                                parent);
    cudaMemsetAsync(root_fp, 0xFF, (size_t)nsq * 4, st);
    cudaMemsetAsync(root_osc, 0xFF, (size_t)nsq * 4, st);
    ucbbr::root_stats_kernel<<<GS, B, 0, st>>>(parent, min_fp, min_osc, nsq, root_fp, root_osc);
    // rank the components (32-bit keys: cell indices, kNone last)
    unsigned int* kfp = reinterpret_cast<unsigned int*>(k_in);
    unsigned int* kosc = reinterpret_cast<unsigned int*>(k_out);
    unsigned int* ids = v_in;
    unsigned int* sorted_keys = head;
    unsigned int* sorted_ids = reinterpret_cast<unsigned int*>(bx);
    ucbbr::rank_keys_kernel<<<GS, B, 0, st>>>(parent, root_fp, root_osc, nsq, kfp, kosc, ids);
    size_t rank_bytes = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, rank_bytes, kfp, sorted_keys, ids, sorted_ids, (int)nsq, 0, 32, st);
    void* rtmp = rank_bytes <= tmp_bytes ? tmp : mem.get<char>(rank_bytes);
    if (!rtmp) {
        err = mem.err;
        return -1;
    }
    cub::DeviceRadixSort::SortPairs(rtmp, rank_bytes, kfp, sorted_keys, ids, sorted_ids, (int)nsq, 0, 32, st);
    ucbbr::assign_rank_kernel<<<GS, B, 0, st>>>(sorted_keys, sorted_ids, nsq, -1, comp_label);
    cub::DeviceRadixSort::SortPairs(rtmp, rank_bytes, kosc, sorted_keys, ids, sorted_ids, (int)nsq, 0, 32, st);
    ucbbr::assign_rank_kernel<<<GS, B, 0, st>>>(sorted_keys, sorted_ids, nsq, 1, comp_label);
    ucbbr::label_kernel<<<G, B, 0, st>>>(order, sq_of, parent, sx, comp_label, N, d_lab);
    if ((ce = cudaGetLastError()) != cudaSuccess) {
        err = std::string("CUDA basins clustering: ") + cudaGetErrorString(ce);
        return -1;
    }
    return 13;  // own kernels (the radix sorts and the scan are CUB's)
}

void label_extremes(const int* labels, long long n, int& mx, int& mn) {
    mx = 0;
    mn = 0;
    for (long long k = 0; k < n; ++k) {
        mx = std::max(mx, labels[k]);
        mn = std::min(mn, labels[k]);
    }
}

bool validate(const ucb_basins_dbscan_request& q, std::string& err) {
    if (!q.krs_body || !*q.krs_body) { err = "krs_body is empty"; return false; }
    if (q.amount_of_x <= 0 || q.amount_of_x > kMaxAmountOfX) { err = "amountOfX out of range"; return false; }
    if (!q.initial_conditions) { err = "initial_conditions.size() != amountOfX"; return false; }
    if (q.n_values > kMaxAmountOfValues) { err = "too many base_values"; return false; }
    if (q.axis_x_var < 0 || q.axis_x_var >= q.amount_of_x) { err = "axis_x_var out of range"; return false; }
    if (q.axis_y_var < 0 || q.axis_y_var >= q.amount_of_x) { err = "axis_y_var out of range"; return false; }
    if (q.axis_x_var == q.axis_y_var) { err = "axis_x_var == axis_y_var (choose different variables)"; return false; }
    if (q.writable_var < -1 || q.writable_var >= q.amount_of_x) { err = "writable_var out of range"; return false; }
    if (q.n_pts <= 0) { err = "n_pts must be > 0"; return false; }
    if (!(q.h > 0.0)) { err = "h must be > 0"; return false; }
    if (!(q.t_max > 0.0)) { err = "t_max must be > 0"; return false; }
    if (q.transient_time < 0) { err = "transient_time must be >= 0"; return false; }
    if (q.pre_scaller <= 0) { err = "pre_scaller must be > 0"; return false; }
    if (!(q.eps_dbscan > 0.0)) { err = "eps_dbscan must be > 0"; return false; }
    if ((long long)q.n_pts * q.n_pts > 0x7FFFFFFFLL) { err = "n_pts too large (n_pts^2 must fit in int)"; return false; }
    return true;
}

CompileRequest features_request(const ucb_basins_dbscan_request& q, SystemCode& sys) {
    SweepMap m;
    m.dim = 2;
    m.par_or_var = 0;
    m.idx[0] = q.axis_x_var;
    m.idx[1] = q.axis_y_var;
    sys = make_system_code(q.krs_body, q.amount_of_x, q.n_values, q.opt.precision, q.opt.mode, false);
    CompileRequest rq;
    rq.name = "ucb_basins_ref.cu";
    std::vector<std::string> defs = clock_defines(sys);
    defs.push_back("UCB_BIF_NO_KERNELS 1");
    // scalar RK4 updates: with the streaming peak finder beside the step, the packed
    // component pairs measured 11 % slower here (FP32 Duffing 1024^2: 987 vs 890 ms)
    defs.push_back("UCB_SCALAR_STEP 1");
    rq.source = make_prelude(q.opt.precision, q.amount_of_x, q.n_values, m, true, sys, defs) +
                "#include \"ucb_device.cuh\"\n#include \"ucb_bif.cuh\"\n#include \"ucb_basins_ref.cuh\"\n";
    rq.headers = device_headers();
    rq.options.push_back(sys.exact ? "--fmad=false" : "--fmad=true");
    rq.kernels = {"ucb_basins_ref_kernel"};
    return rq;
}

// Per-field min / max of run_basins: finite values other than the 999 / -999 sentinels.
void minmax_features(const double* v, long long n, double& mn, double& mx) {
    mn = std::numeric_limits<double>::infinity();
    mx = -mn;
    for (long long k = 0; k < n; ++k) {
        const double x = v[k];
        if (!std::isfinite(x) || x == 999.0 || x == -999.0) continue;
        mn = std::min(mn, x);
        mx = std::max(mx, x);
    }
    if (!std::isfinite(mn) || !std::isfinite(mx)) mn = mx = 0.0;
}

}  // namespace
}  // namespace ucb

using namespace ucb;

extern "C" int ucb_precompile_basins_dbscan(const ucb_basins_dbscan_request* req, char* err_out, int err_len) {
    std::string err;
    if (!req || !validate(*req, err)) {
        if (err_out && err_len > 0) std::snprintf(err_out, (size_t)err_len, "%s", err.c_str());
        return UCB_E_INVALID;
    }
    SystemCode sys;
    CompileRequest rq = features_request(*req, sys);
    TuneConfig shape;
    if (!tune_request(nullptr, req->opt, 128, rq, shape, err)) {
        if (err_out && err_len > 0) std::snprintf(err_out, (size_t)err_len, "%s", err.c_str());
        return UCB_E_INVALID;
    }
    if (!precompile_to_disk(rq, err)) {
        if (err_out && err_len > 0) std::snprintf(err_out, (size_t)err_len, "%s", err.c_str());
        return UCB_E_COMPILE;
    }
    if (err_out && err_len > 0) std::snprintf(err_out, (size_t)err_len, "%s", sys.note.c_str());
    return UCB_OK;
}

extern "C" int ucb_run_basins_dbscan(ucb_engine* e, const ucb_basins_dbscan_request* req,
                                     ucb_basins_dbscan_result* res) {
    if (!e || !req || !res) return UCB_E_INVALID;
    const ucb_basins_dbscan_request& q = *req;
    res->ok = res->cancelled = 0;
    res->error[0] = 0;
    res->kernel_ms = res->cluster_ms = 0;
    res->steps = 0;
    std::string err;
    if (!validate(q, err)) return fail(e, res, UCB_E_INVALID, err);
    if (!res->labels || !res->avg_peaks || !res->avg_intervals || !res->classes)
        return fail(e, res, UCB_E_INVALID, "result buffers are NULL");
    if (q.cancel && *q.cancel) {
        res->cancelled = 1;
        return fail(e, res, UCB_E_CANCELLED, "Cancelled by user");
    }
    const int prec = q.opt.precision;
    const long long points = (long long)(q.t_max / q.h / q.pre_scaller);
    const long long skip = (long long)(q.transient_time / q.h);
    if (points <= 0) return fail(e, res, UCB_E_INVALID, "computed amountOfPointsInBlock <= 0");
    if (!ensure_init(e, err)) return fail(e, res, UCB_E_NOGPU, err);
    SystemCode sys;
    CompileRequest rq = features_request(q, sys);
    TuneConfig shape;
    if (!tune_request(e, q.opt, 128, rq, shape, err)) return fail(e, res, UCB_E_INVALID, err);
    auto mod = e->modules.get(rq, err);
    if (!mod) return fail(e, res, UCB_E_COMPILE, err);
    CUfunction fn = mod->functions["ucb_basins_ref_kernel"];

    const int n = q.n_pts;
    const long long total = (long long)n * n;
    cudaStream_t st = e->stream;
    std::vector<double> t0d, t1d;
    std::vector<float> t0f, t1f;
    axis_table(prec, n, q.axis_x_lo, q.axis_x_hi, false, t0d, t0f);
    axis_table(prec, n, q.axis_y_lo, q.axis_y_hi, false, t1d, t1f);
    const size_t esz = prec == UCB_PREC_F64 ? 8 : 4;
    const size_t tab_bytes = (size_t)n * esz;
    const size_t off0 = 256, off1 = 256 + ((tab_bytes + 255) / 256) * 256;
    if (!ensure_workspace(e, off1 + tab_bytes + 256, err)) return fail(e, res, UCB_E_CUDA, err);
    char* ws = static_cast<char*>(e->ws);
    DeviceArena mem{e, st, {}, {}};
    double* d_f1 = mem.get<double>(total);
    double* d_f2 = mem.get<double>(total);
    int* d_cls = mem.get<int>(total);
    int* d_lab = mem.get<int>(total);
    if (!d_f1 || !d_f2 || !d_cls || !d_lab) return fail(e, res, UCB_E_CUDA, mem.err);
    cudaMemcpyAsync(ws + off0, prec == UCB_PREC_F64 ? (const void*)t0d.data() : (const void*)t0f.data(), tab_bytes,
                    cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(ws + off1, prec == UCB_PREC_F64 ? (const void*)t1d.data() : (const void*)t1f.data(), tab_bytes,
                    cudaMemcpyHostToDevice, st);
    cudaMemsetAsync(ws, 0, 16, st);
    if (q.progress_phase) *q.progress_phase = 1;
    if (q.progress) *q.progress = 0.0f;
    // 1. classes and features (UcbBasinsRefParams field by field)
    ParamPack pk;
    pk.put<long long>(total);
    pk.put<int>(n);
    pk.put<int>(q.pre_scaller);
    pk.put<int>(q.writable_var);
    pk.put<int>(q.feature1);
    pk.put<int>(q.feature2);
    pk.put<int>(0);
    pk.put<long long>(skip);
    pk.put<long long>(points);
    for (double v : {q.h, q.max_value, q.mult1, q.mult2, q.h * (double)q.pre_scaller}) pk.put_numb(prec, v);
    for (int i = 0; i < q.amount_of_x; ++i) pk.put_numb(prec, q.initial_conditions[i]);
    for (int i = 0; i < std::max(q.n_values, 1); ++i) pk.put_numb(prec, i < q.n_values ? q.base_values[i] : 0.0);
    pk.put<const void*>(ws + off0);
    pk.put<const void*>(ws + off1);
    pk.put<void*>(d_f1);
    pk.put<void*>(d_f2);
    pk.put<void*>(d_cls);
    pk.put<void*>(ws);
    pk.put<void*>(ws + 8);
    EventPair cev;
    begin_run(e);
    cudaEventRecord(e->ev0, st);
    if (!launch_packed(e, fn, persistent_grid(e, fn, shape.block, total), shape.block, st, pk, err))
        return fail(e, res, UCB_E_CUDA, err);
    cudaEventRecord(e->ev1, st);
    {
        const int wr = wait_run(e, e->ev1, q.cancel, q.progress, total, err);
        if (wr == UCB_E_CANCELLED) res->cancelled = 1;
        if (wr != UCB_OK) return fail(e, res, wr, err);
    }

    // 2. clustering of the features
    if (q.cancel && *q.cancel) {
        res->cancelled = 1;
        return fail(e, res, UCB_E_CANCELLED, "Cancelled by user");
    }
    if (q.progress_phase) *q.progress_phase = 2;
    if (q.progress) *q.progress = 0.0f;
    cudaEventRecord(cev.a, st);
    const int nl = cluster_features(e, st, mem, d_f1, d_f2, d_cls, (unsigned int)total, q.eps_dbscan,
                                    prec == UCB_PREC_F32 ? 1 : 0, d_lab, err);
    if (nl < 0) return fail(e, res, UCB_E_CUDA, err);
    e->launches += nl;
    cudaEventRecord(cev.b, st);
    unsigned long long steps = 0;
    cudaError_t ce;
    if ((ce = cudaMemcpyAsync(res->labels, d_lab, (size_t)total * 4, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (ce = cudaMemcpyAsync(res->avg_peaks, d_f1, (size_t)total * 8, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (ce = cudaMemcpyAsync(res->avg_intervals, d_f2, (size_t)total * 8, cudaMemcpyDeviceToHost, st)) !=
            cudaSuccess ||
        (ce = cudaMemcpyAsync(res->classes, d_cls, (size_t)total * 4, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (ce = cudaMemcpyAsync(&steps, ws + 8, 8, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (ce = cudaStreamSynchronize(st)) != cudaSuccess)
        return fail(e, res, UCB_E_CUDA, std::string("CUDA basins: ") + cudaGetErrorString(ce));
    float ms = 0, cms = 0;
    cudaEventElapsedTime(&ms, e->ev0, e->ev1);
    cudaEventElapsedTime(&cms, cev.a, cev.b);
    res->kernel_ms = ms;
    res->cluster_ms = cms;
    res->steps = (long long)steps;
    label_extremes(res->labels, total, res->n_clusters, res->min_cluster_idx);
    minmax_features(res->avg_peaks, total, res->avg_peaks_min, res->avg_peaks_max);
    minmax_features(res->avg_intervals, total, res->avg_intervals_min, res->avg_intervals_max);
    res->n_pts = n;
    if (q.csv_output_path && *q.csv_output_path) {
        const csv::Common cc = csv::common(q.base_values, q.n_values, q.initial_conditions, q.amount_of_x,
                                           q.opt.precision == UCB_PREC_F32);
        csv::basins(q.csv_output_path, cc, q.t_max, q.transient_time, q.h, q.pre_scaller, q.eps_dbscan,
                    q.writable_var, q.axis_x_var, q.axis_y_var, q.axis_x_lo, q.axis_x_hi, q.axis_y_lo, q.axis_y_hi, n,
                    res->labels, res->avg_peaks, res->avg_intervals, res->classes);
    }
    if (q.progress) *q.progress = 1.0f;
    res->ok = 1;
    return UCB_OK;
}

extern "C" int ucb_run_basins_recluster(ucb_engine* e, const ucb_basins_recluster_request* req,
                                        ucb_basins_recluster_result* res) {
    if (!e || !req || !res) return UCB_E_INVALID;
    const ucb_basins_recluster_request& q = *req;
    res->ok = res->cancelled = 0;
    res->error[0] = 0;
    res->cluster_ms = 0;
    // validation of run_basins_recluster (parametric_engine.cpp:6528-6535)
    if (!q.krs_body || !*q.krs_body) return fail(e, res, UCB_E_INVALID, "krs_body is empty");
    if (q.amount_of_x <= 0 || q.amount_of_x > kMaxAmountOfX)
        return fail(e, res, UCB_E_INVALID, "amountOfX out of range");
    if (q.n_pts <= 0) return fail(e, res, UCB_E_INVALID, "n_pts must be > 0");
    if (!(q.eps_dbscan > 0.0)) return fail(e, res, UCB_E_INVALID, "eps_dbscan must be > 0");
    if ((long long)q.n_pts * q.n_pts > 0x7FFFFFFFLL)
        return fail(e, res, UCB_E_INVALID, "n_pts too large (n_pts^2 must fit in int)");
    if (!q.avg_peaks) return fail(e, res, UCB_E_INVALID, "avg_peaks: size does not match n_pts^2");
    if (!q.avg_intervals) return fail(e, res, UCB_E_INVALID, "avg_intervals: size does not match n_pts^2");
    if (!q.classes) return fail(e, res, UCB_E_INVALID, "helpful_array: size does not match n_pts^2");
    if (!res->labels) return fail(e, res, UCB_E_INVALID, "result buffers are NULL");
    if (q.cancel && *q.cancel) {
        res->cancelled = 1;
        return fail(e, res, UCB_E_CANCELLED, "Cancelled by user");
    }
    std::string err;
    if (!ensure_init(e, err)) return fail(e, res, UCB_E_NOGPU, err);
    const long long total = (long long)q.n_pts * q.n_pts;
    cudaStream_t st = e->stream;
    DeviceArena mem{e, st, {}, {}};
    double* d_f1 = mem.get<double>(total);
    double* d_f2 = mem.get<double>(total);
    int* d_cls = mem.get<int>(total);
    int* d_lab = mem.get<int>(total);
    if (!d_f1 || !d_f2 || !d_cls || !d_lab) return fail(e, res, UCB_E_CUDA, mem.err);
    cudaMemcpyAsync(d_f1, q.avg_peaks, (size_t)total * 8, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(d_f2, q.avg_intervals, (size_t)total * 8, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(d_cls, q.classes, (size_t)total * 4, cudaMemcpyHostToDevice, st);
    if (q.progress) *q.progress = 0.0f;
    EventPair cev;
    cudaEventRecord(cev.a, st);
    const int nl = cluster_features(e, st, mem, d_f1, d_f2, d_cls, (unsigned int)total, q.eps_dbscan,
                                    q.opt.precision == UCB_PREC_F32 ? 1 : 0, d_lab, err);
    if (nl < 0) return fail(e, res, UCB_E_CUDA, err);
    e->launches += nl;
    cudaEventRecord(cev.b, st);
    cudaError_t ce;
    if ((ce = cudaMemcpyAsync(res->labels, d_lab, (size_t)total * 4, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (ce = cudaStreamSynchronize(st)) != cudaSuccess)
        return fail(e, res, UCB_E_CUDA, std::string("CUDA basins recluster: ") + cudaGetErrorString(ce));
    float cms = 0;
    cudaEventElapsedTime(&cms, cev.a, cev.b);
    res->cluster_ms = cms;
    label_extremes(res->labels, total, res->n_clusters, res->min_cluster_idx);
    res->n_pts = q.n_pts;
    if (q.progress) *q.progress = 1.0f;
    res->ok = 1;
    return UCB_OK;
}
