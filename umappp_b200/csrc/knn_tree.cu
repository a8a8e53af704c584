// Tile pruning for the exact tensor-core kNN: a spatial ordering of the
// points and, per block of queries, the reference tiles that can hold one of
// its neighbours.
//
// Ordering (random-projection tree): the points of every instance are split
// recursively -- projected on the difference of two of the segment's own
// points, sorted by the projection, cut so that the left part is a whole
// number of 128-row tiles -- until each segment is one tile.  Clustered data
// (single-cell profiles, mixtures) then come out with tiles that each sit in
// one cluster.
//
// Bounds: every 128-row reference tile T and every query block B (the rows one
// CTA of the search serves) gets a centroid c (FP32) and a radius R (an upper
// bound of |x - c| over its points, FP64 rounded up).  For a query q in B and a
// point r in T the triangle inequality gives
//     |q - r| >= |c_B - c_T| - R_B - R_T =: lb(B, T),
// and every query of B has at least (|B| - 1) other points of B within 2 R_B.
// If |B| - 1 >= k, the k-th neighbour of q is therefore within 2 R_B, and a
// tile with lb(B, T) > 2 R_B cannot hold any of q's k nearest neighbours: it
// is left out of B's list.  This is exact (no neighbour is lost); for data
// without cluster structure the lists simply cover every tile.
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

#include "stages.cuh"

namespace umapb {

namespace {

constexpr int TREE_LEAF = 128;

// Projection key of every position: the point's coordinates dotted with the
// difference of two points of its segment; 0 in segments that are leaves.
__global__ void rp_keys_kernel(const float* __restrict__ data, int32_t dim, int32_t n,
                               const int32_t* __restrict__ perm, int32_t nseg, const int32_t* __restrict__ seg_start,
                               const int32_t* __restrict__ seg_a, const int32_t* __restrict__ seg_b,
                               float* __restrict__ keys) {
    for (int32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        int lo = 0, hi = nseg - 1;   // segment of position p: last start <= p
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (seg_start[mid] <= p) lo = mid; else hi = mid - 1;
        }
        const int32_t a = seg_a[lo], b = seg_b[lo];
        float key = 0.0f;
        if (a >= 0) {
            const float* x = data + static_cast<size_t>(perm[p]) * dim;
            const float* xa = data + static_cast<size_t>(perm[a]) * dim;
            const float* xb = data + static_cast<size_t>(perm[b]) * dim;
            for (int d = 0; d < dim; ++d) key = fmaf(x[d], xa[d] - xb[d], key);
        }
        keys[p] = key;
    }
}

__global__ void iota_kernel(int32_t* __restrict__ v, int32_t n) {
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) v[i] = i;
}

// out[i] = row_map[idx[i]] (or -1 where idx[i] < 0)
__global__ void gather_rows_kernel(const int32_t* __restrict__ idx, size_t count, const int32_t* __restrict__ row_map,
                                   int32_t* __restrict__ out) {
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < count; i += size_t(gridDim.x) * blockDim.x)
        out[i] = idx[i] >= 0 ? row_map[idx[i]] : -1;
}

__global__ void pad_order_kernel(const int32_t* __restrict__ perm, int32_t ninst, const int32_t* __restrict__ inst,
                                 const int32_t* __restrict__ pad_start, int32_t n_pad, int32_t* __restrict__ row_map) {
    for (int32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < n_pad; r += gridDim.x * blockDim.x) {
        int lo = 0, hi = ninst - 1;   // instance whose padded range holds r
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (pad_start[mid] <= r) lo = mid; else hi = mid - 1;
        }
        const int32_t off = r - pad_start[lo];
        row_map[r] = (off < inst[lo + 1] - inst[lo]) ? perm[inst[lo] + off] : -1;
    }
}

// Centroid, radius and real-row count of every group of 'rows' operand rows.
__global__ void group_bounds_kernel(const float* __restrict__ data, int32_t dim, const int32_t* __restrict__ row_map,
                                    int32_t rows, float* __restrict__ centroid, float* __restrict__ radius,
                                    int32_t* __restrict__ count) {
    const int32_t g = blockIdx.x;
    const int32_t r0 = g * rows;
    __shared__ double red[256];
    __shared__ int cnt;
    if (threadIdx.x == 0) cnt = 0;
    __syncthreads();
    int c = 0;
    for (int r = threadIdx.x; r < rows; r += blockDim.x) c += (row_map[r0 + r] >= 0);
    atomicAdd(&cnt, c);
    __syncthreads();
    const int m = cnt;
    float* cg = centroid + static_cast<size_t>(g) * dim;
    for (int d = threadIdx.x; d < dim; d += blockDim.x) {
        double s = 0;
        for (int r = 0; r < rows; ++r) {
            const int32_t src = row_map[r0 + r];
            if (src >= 0) s += data[static_cast<size_t>(src) * dim + d];
        }
        cg[d] = m ? static_cast<float>(s / m) : 0.0f;
    }
    __syncthreads();
    double worst = 0;
    for (int r = threadIdx.x; r < rows; r += blockDim.x) {
        const int32_t src = row_map[r0 + r];
        if (src < 0) continue;
        double s = 0;
        for (int d = 0; d < dim; ++d) {
            const double v = static_cast<double>(data[static_cast<size_t>(src) * dim + d]) - cg[d];
            s += v * v;
        }
        worst = fmax(worst, s);
    }
    red[threadIdx.x] = worst;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + w]);
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        // rounded up, with a margin for the FP64 sum
        radius[g] = __double2float_ru(sqrt(red[0]) * (1.0 + 1e-9) + 1e-30);
        count[g] = m;
    }
}

// Whether reference tile t may hold a neighbour of a query in block b.
__device__ __forceinline__ bool tile_needed(const float* __restrict__ cb, float rb, const float* __restrict__ ct,
                                            float rt, int dim) {
    double s = 0;
    for (int d = 0; d < dim; ++d) {
        const double v = static_cast<double>(cb[d]) - ct[d];
        s += v * v;
    }
    const double lb = sqrt(s) * (1.0 - 1e-9) - rb - rt;
    return lb <= 2.0 * rb;
}

// One warp per query block: count (write == false) or write the indices of
// the reference tiles of its instance that it needs, in ascending order.
__global__ void tile_lists_kernel(int32_t nblocks, int32_t block_rows, const int32_t* __restrict__ blk_tile0,
                                  const int32_t* __restrict__ blk_ntiles, const float* __restrict__ bc,
                                  const float* __restrict__ br, const int32_t* __restrict__ bcount,
                                  const float* __restrict__ tc, const float* __restrict__ tr, int32_t dim, int32_t k,
                                  bool prune, const int64_t* __restrict__ offsets, int32_t* __restrict__ counts,
                                  int32_t* __restrict__ lists) {
    const int lane = threadIdx.x & 31;
    const int32_t b = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (b >= nblocks) return;
    const int32_t t0 = blk_tile0[b], nt = blk_ntiles[b];
    const bool all = !prune || bcount[b] < k + 1;
    const float* cb = bc + static_cast<size_t>(b) * dim;
    const float rb = br[b];
    int64_t out = lists ? offsets[b] : 0;
    int32_t total = 0;
    for (int32_t base = 0; base < nt; base += 32) {
        const int32_t t = t0 + base + lane;
        bool need = false;
        if (base + lane < nt) need = all || tile_needed(cb, rb, tc + static_cast<size_t>(t) * dim, tr[t], dim);
        const unsigned m = __ballot_sync(0xffffffffu, need);
        if (lists && need) lists[out + __popc(m & ((1u << lane) - 1u))] = t;
        out += __popc(m);
        total += __popc(m);
    }
    if (!lists && lane == 0) counts[b] = total;
}

}  // namespace

void knn_tree_order(const float* data, int32_t dim, const std::vector<int32_t>& inst, bool tree, KnnTiles& out,
                    cudaStream_t s) {
    const int ninst = static_cast<int>(inst.size()) - 1;
    const int32_t n = inst[ninst];
    out.pad_start.assign(ninst + 1, 0);
    for (int i = 0; i < ninst; ++i) {
        const int32_t len = inst[i + 1] - inst[i];
        out.pad_start[i + 1] = out.pad_start[i] + ((len + TREE_LEAF - 1) / TREE_LEAF) * TREE_LEAF;
    }
    out.n_pad = std::max(out.pad_start[ninst], TREE_LEAF);
    DevArray<int32_t> perm(n, s), perm2(n, s);
    DevArray<float> keys(n, s), keys2(n, s);
    iota_kernel<<<grid_for(n, 256), 256, 0, s>>>(perm.get(), n);
    UMAPB_LAUNCH_CHECK();

    // segments over positions of perm; the instances to begin with
    std::vector<int32_t> st(inst.begin(), inst.end() - 1), len(ninst);
    for (int i = 0; i < ninst; ++i) len[i] = inst[i + 1] - inst[i];
    uint64_t h = 0x9E3779B97F4A7C15ull;
    auto next = [&h]() {   // splitmix64: the choice of the two direction points
        uint64_t z = (h += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    };
    DevArray<int32_t> d_start, d_end, d_a, d_b;
    for (int level = 0; tree && level < 40; ++level) {
        const int nseg = static_cast<int>(st.size());
        std::vector<int32_t> a(nseg, -1), b(nseg, -1), en(nseg);
        bool any = false;
        for (int g = 0; g < nseg; ++g) {
            en[g] = st[g] + len[g];
            if (len[g] > TREE_LEAF) {
                any = true;
                a[g] = st[g] + static_cast<int32_t>(next() % static_cast<uint64_t>(len[g]));
                b[g] = st[g] + static_cast<int32_t>(next() % static_cast<uint64_t>(len[g]));
            }
        }
        if (!any) break;
        d_start.reserve(nseg, s);
        d_end.reserve(nseg, s);
        d_a.reserve(nseg, s);
        d_b.reserve(nseg, s);
        UMAPB_CUDA(cudaMemcpyAsync(d_start.get(), st.data(), nseg * sizeof(int32_t), cudaMemcpyHostToDevice, s));
        UMAPB_CUDA(cudaMemcpyAsync(d_end.get(), en.data(), nseg * sizeof(int32_t), cudaMemcpyHostToDevice, s));
        UMAPB_CUDA(cudaMemcpyAsync(d_a.get(), a.data(), nseg * sizeof(int32_t), cudaMemcpyHostToDevice, s));
        UMAPB_CUDA(cudaMemcpyAsync(d_b.get(), b.data(), nseg * sizeof(int32_t), cudaMemcpyHostToDevice, s));
        rp_keys_kernel<<<grid_for(n, 256), 256, 0, s>>>(data, dim, n, perm.get(), nseg, d_start.get(), d_a.get(),
                                                        d_b.get(), keys.get());
        UMAPB_LAUNCH_CHECK();
        size_t tb = 0;
        UMAPB_CUDA(cub::DeviceSegmentedSort::SortPairs(nullptr, tb, keys.get(), keys2.get(), perm.get(), perm2.get(), n,
                                                       nseg, d_start.get(), d_end.get(), s));
        {
            DevArray<unsigned char> temp(tb, s);
            UMAPB_CUDA(cub::DeviceSegmentedSort::SortPairs(temp.get(), tb, keys.get(), keys2.get(), perm.get(),
                                                           perm2.get(), n, nseg, d_start.get(), d_end.get(), s));
        }
        std::swap(perm, perm2);
        UMAPB_SYNC(s);   // the host segment tables are the copies' sources
        std::vector<int32_t> st2, len2;
        st2.reserve(2 * nseg);
        len2.reserve(2 * nseg);
        for (int g = 0; g < nseg; ++g) {
            if (len[g] > TREE_LEAF) {
                const int32_t tiles = (len[g] + TREE_LEAF - 1) / TREE_LEAF;
                const int32_t left = (tiles + 1) / 2 * TREE_LEAF;
                st2.push_back(st[g]);
                len2.push_back(left);
                st2.push_back(st[g] + left);
                len2.push_back(len[g] - left);
            } else {
                st2.push_back(st[g]);
                len2.push_back(len[g]);
            }
        }
        st.swap(st2);
        len.swap(len2);
    }
    DevArray<int32_t> d_inst(inst.size(), s), d_pad(out.pad_start.size(), s);
    UMAPB_CUDA(cudaMemcpyAsync(d_inst.get(), inst.data(), inst.size() * sizeof(int32_t), cudaMemcpyHostToDevice, s));
    UMAPB_CUDA(cudaMemcpyAsync(d_pad.get(), out.pad_start.data(), out.pad_start.size() * sizeof(int32_t),
                               cudaMemcpyHostToDevice, s));
    out.row_map.allocate(out.n_pad, s);
    pad_order_kernel<<<grid_for(out.n_pad, 256), 256, 0, s>>>(perm.get(), ninst, d_inst.get(), d_pad.get(), out.n_pad,
                                                              out.row_map.get());
    UMAPB_LAUNCH_CHECK();
    UMAPB_SYNC(s);   // host vectors above
}

void knn_tile_tasks(const float* data, int32_t dim, const KnnTiles& t, const std::vector<int32_t>& inst, int qt,
                    int32_t k, bool prune, KnnTasks& out, cudaStream_t s) {
    const int ninst = static_cast<int>(inst.size()) - 1;
    const int32_t block_rows = TREE_LEAF * qt;
    const int32_t ntiles = t.n_pad / TREE_LEAF;
    // query blocks: qt tiles each, never across an instance boundary
    std::vector<int32_t> qbase, qlimit, tile0, ntl;
    for (int i = 0; i < ninst; ++i) {
        const int32_t p0 = t.pad_start[i], p1 = t.pad_start[i + 1];
        for (int32_t r = p0; r < p1; r += block_rows) {
            qbase.push_back(r);
            qlimit.push_back(p0 + (inst[i + 1] - inst[i]));
            tile0.push_back(p0 / TREE_LEAF);
            ntl.push_back((p1 - p0) / TREE_LEAF);
        }
    }
    const int32_t nb = static_cast<int32_t>(qbase.size());
    // bounds of the reference tiles and of the query blocks (a block may run
    // into the next instance's rows; those rows are excluded by its own map)
    DevArray<float> tcen(static_cast<size_t>(ntiles) * dim, s), trad(ntiles, s), bcen(static_cast<size_t>(nb) * dim, s),
        brad(nb, s);
    DevArray<int32_t> tcnt(ntiles, s), bcnt(nb, s);
    group_bounds_kernel<<<ntiles, 128, 0, s>>>(data, dim, t.row_map.get(), TREE_LEAF, tcen.get(), trad.get(), tcnt.get());
    UMAPB_LAUNCH_CHECK();
    // a query block's rows: its own map entries, cut at its instance's end
    DevArray<int32_t> bmap(static_cast<size_t>(nb) * block_rows, s);
    {
        std::vector<int32_t> idx(static_cast<size_t>(nb) * block_rows);
        for (int32_t b = 0; b < nb; ++b)
            for (int32_t r = 0; r < block_rows; ++r) {
                const int32_t row = qbase[b] + r;
                idx[static_cast<size_t>(b) * block_rows + r] = (row < qlimit[b]) ? row : -1;
            }
        DevArray<int32_t> d_idx(idx.size(), s);
        UMAPB_CUDA(cudaMemcpyAsync(d_idx.get(), idx.data(), idx.size() * sizeof(int32_t), cudaMemcpyHostToDevice, s));
        gather_rows_kernel<<<grid_for(idx.size(), 256), 256, 0, s>>>(d_idx.get(), idx.size(), t.row_map.get(),
                                                                     bmap.get());
        UMAPB_LAUNCH_CHECK();
        UMAPB_SYNC(s);
    }
    group_bounds_kernel<<<nb, 128, 0, s>>>(data, dim, bmap.get(), block_rows, bcen.get(), brad.get(), bcnt.get());
    UMAPB_LAUNCH_CHECK();

    DevArray<int32_t> d_tile0(nb, s), d_ntl(nb, s), counts(nb, s);
    DevArray<int64_t> offsets(nb + 1, s);
    UMAPB_CUDA(cudaMemcpyAsync(d_tile0.get(), tile0.data(), nb * sizeof(int32_t), cudaMemcpyHostToDevice, s));
    UMAPB_CUDA(cudaMemcpyAsync(d_ntl.get(), ntl.data(), nb * sizeof(int32_t), cudaMemcpyHostToDevice, s));
    const unsigned warps_grid = static_cast<unsigned>((static_cast<int64_t>(nb) * 32 + 255) / 256);
    tile_lists_kernel<<<warps_grid, 256, 0, s>>>(nb, block_rows, d_tile0.get(), d_ntl.get(), bcen.get(), brad.get(),
                                                 bcnt.get(), tcen.get(), trad.get(), dim, k, prune, nullptr,
                                                 counts.get(), nullptr);
    UMAPB_LAUNCH_CHECK();
    std::vector<int32_t> hc(nb);
    UMAPB_CUDA(cudaMemcpyAsync(hc.data(), counts.get(), nb * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    UMAPB_SYNC(s);
    std::vector<int64_t> ho(nb + 1, 0);
    for (int32_t b = 0; b < nb; ++b) ho[b + 1] = ho[b] + hc[b];
    out.total_tiles = ho[nb];
    out.tile_list.allocate(std::max<int64_t>(ho[nb], 1), s);
    UMAPB_CUDA(cudaMemcpyAsync(offsets.get(), ho.data(), (nb + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, s));
    tile_lists_kernel<<<warps_grid, 256, 0, s>>>(nb, block_rows, d_tile0.get(), d_ntl.get(), bcen.get(), brad.get(),
                                                 bcnt.get(), tcen.get(), trad.get(), dim, k, prune, offsets.get(),
                                                 counts.get(), out.tile_list.get());
    UMAPB_LAUNCH_CHECK();
    // tasks, longest lists first (they are scheduled first and finish together)
    std::vector<int32_t> order(nb);
    for (int32_t b = 0; b < nb; ++b) order[b] = b;
    std::stable_sort(order.begin(), order.end(), [&](int32_t x, int32_t y) { return hc[x] > hc[y]; });
    std::vector<int4> tasks(nb);
    for (int32_t j = 0; j < nb; ++j) {
        const int32_t b = order[j];
        require(ho[b] <= INT32_MAX, "tile lists too long", UMAPB_ERR_OVERFLOW);
        tasks[j] = make_int4(qbase[b], static_cast<int32_t>(ho[b]), hc[b], qlimit[b]);
    }
    out.count = nb;
    out.tasks.allocate(nb, s);
    UMAPB_CUDA(cudaMemcpyAsync(out.tasks.get(), tasks.data(), nb * sizeof(int4), cudaMemcpyHostToDevice, s));
    UMAPB_SYNC(s);   // host vectors above
}

}  // namespace umapb
