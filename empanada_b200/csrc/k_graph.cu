// k_graph.cu -- the unitig layer over output.bin: the downstream consumer of
// the overlap edges (the reference writes only the edge records; its GFA
// writers, overlap.cu:129-190, are dead code).
//
// Nodes are read-ends (rid = 2i read i, 2i+1 its reverse complement), edges
// the records' (from, to) pairs: the suffix of `from` equals the prefix of
// `to` over ovlp_len bases.  Under the reference's remove_used rule every
// suffix keeps only its longest overlaps, so no edge is transitive (u -> v
// and u -> w share one length) and the graph needs no reduction.  A unitig is
// a maximal path of edges u -> v with out-degree(u) = in-degree(v) = 1; a
// cycle of such edges is cut before its smallest node.  Every node belongs
// to exactly one unitig (a node on no such edge is a unitig of one).
//
//   scatter   the records' edges into (from, to) arrays
//   degree    in- and out-degree of every node
//   link      succ / pred along the unitig edges
//   walk      one thread per head (a node without pred) follows succ and
//             gives each node of its path the head and the distance to it;
//             the nodes no walk reaches lie on cycles
//   cycles    the smallest node of every cycle by doubling over pred (only
//             cycle nodes take part); the cycle is cut before it and walked
//             from it
//   place     unitig sizes at their heads, starts by a scan, each node at
//             start(head) + distance
#include "kernels.h"

namespace emp {
namespace {

constexpr uint32_t kNone = 0xffffffffu;
constexpr int kGT = 256;

__global__ void graph_scatter_kernel(const uint8_t *__restrict__ out, const uint64_t *__restrict__ rec_off,
                                     const uint64_t *__restrict__ rec_e0, uint32_t nrec, uint64_t E,
                                     uint32_t *__restrict__ from, uint32_t *__restrict__ to) {
    for (uint64_t e = (uint64_t)blockIdx.x * kGT + threadIdx.x; e < E; e += (uint64_t)gridDim.x * kGT) {
        uint32_t lo = 0, hi = nrec;  // last record whose first edge is <= e
        while (hi - lo > 1) {
            const uint32_t m = (lo + hi) >> 1;
            if (rec_e0[m] <= e) lo = m;
            else hi = m;
        }
        const uint64_t k = e - rec_e0[lo], n = rec_e0[lo + 1] - rec_e0[lo];
        const uint8_t *r = out + rec_off[lo] + 12;  // u64 n, i32 ovlp_len, u32 from[n], u32 to[n]
        uint32_t f, t;
        memcpy(&f, r + 4 * k, 4);
        memcpy(&t, r + 4 * (n + k), 4);
        from[e] = f;
        to[e] = t;
    }
}

__global__ void graph_degree_kernel(const uint32_t *__restrict__ from, const uint32_t *__restrict__ to, uint64_t E,
                                    uint32_t nodes, uint32_t *__restrict__ dout, uint32_t *__restrict__ din,
                                    uint32_t *err) {
    for (uint64_t e = (uint64_t)blockIdx.x * kGT + threadIdx.x; e < E; e += (uint64_t)gridDim.x * kGT) {
        const uint32_t u = from[e], v = to[e];
        if (u >= nodes || v >= nodes) {
            atomicOr(err, kErrCapacity);  // an edge names a read-end beyond the reads given
            continue;
        }
        atomicAdd(dout + u, 1u);
        atomicAdd(din + v, 1u);
    }
}

__global__ void graph_link_kernel(const uint32_t *__restrict__ from, const uint32_t *__restrict__ to, uint64_t E,
                                  uint32_t nodes, const uint32_t *__restrict__ dout, const uint32_t *__restrict__ din,
                                  uint32_t *__restrict__ succ, uint32_t *__restrict__ pred) {
    for (uint64_t e = (uint64_t)blockIdx.x * kGT + threadIdx.x; e < E; e += (uint64_t)gridDim.x * kGT) {
        const uint32_t u = from[e], v = to[e];
        if (u >= nodes || v >= nodes) continue;
        if (dout[u] == 1 && din[v] == 1) {
            succ[u] = v;
            pred[v] = u;
        }
    }
}

// One thread per head h (pred[h] == none, or a cycle's smallest node once
// `cyc` is set): every node of its path gets hop = h and its distance.
__global__ void graph_walk_kernel(const uint32_t *__restrict__ pred, const uint32_t *__restrict__ succ,
                                  const uint32_t *__restrict__ mn, uint32_t nodes, int cyc, uint32_t *__restrict__ hop,
                                  uint32_t *__restrict__ dist) {
    for (uint32_t h = blockIdx.x * kGT + threadIdx.x; h < nodes; h += gridDim.x * kGT) {
        if (cyc ? (hop[h] != kNone || mn[h] != h) : pred[h] != kNone) continue;
        uint32_t x = h, d = 0;
        do {
            hop[x] = h;
            dist[x] = d++;
            x = succ[x];
        } while (x != kNone && x != h && d <= nodes);
    }
}

// Cycle minimum by doubling over pred: mn/nx in, mn2/nx2 out (nodes whose
// hop reached a head are not on a cycle and are left alone).
__global__ void graph_cycle_min_kernel(const uint32_t *__restrict__ hop, const uint32_t *__restrict__ mn,
                                       const uint32_t *__restrict__ nx, uint32_t nodes, uint32_t *__restrict__ mn2,
                                       uint32_t *__restrict__ nx2) {
    for (uint32_t u = blockIdx.x * kGT + threadIdx.x; u < nodes; u += gridDim.x * kGT) {
        if (hop[u] != kNone) continue;  // on a path
        const uint32_t x = nx[u];
        mn2[u] = min(mn[u], mn[x]);
        nx2[u] = nx[x];
    }
}

// Cut every cycle before its smallest node c: pred[c] and succ[pred[c]] cleared.
__global__ void graph_cut_kernel(const uint32_t *__restrict__ hop, const uint32_t *__restrict__ mn, uint32_t nodes,
                                 uint32_t *__restrict__ pred, uint32_t *__restrict__ succ, uint32_t *cycles) {
    for (uint32_t u = blockIdx.x * kGT + threadIdx.x; u < nodes; u += gridDim.x * kGT) {
        if (hop[u] != kNone) continue;  // on a path
        const uint32_t p = pred[u];
        if (mn[u] == u) {
            succ[p] = kNone;
            pred[u] = kNone;
            atomicAdd(cycles, 1u);
        }
    }
}

__global__ void graph_size_kernel(const uint32_t *__restrict__ hop, uint32_t nodes, uint32_t *__restrict__ size) {
    for (uint32_t u = blockIdx.x * kGT + threadIdx.x; u < nodes; u += gridDim.x * kGT) atomicAdd(size + hop[u], 1u);
}

__global__ void graph_place_kernel(const uint32_t *__restrict__ hop, const uint32_t *__restrict__ dist,
                                   const uint64_t *__restrict__ start, uint32_t nodes, uint32_t *__restrict__ order) {
    for (uint32_t u = blockIdx.x * kGT + threadIdx.x; u < nodes; u += gridDim.x * kGT)
        order[start[hop[u]] + dist[u]] = u;
}

unsigned grid_of(uint64_t n) {
    const uint64_t g = (n + kGT - 1) / kGT;
    return (unsigned)(g < 1 ? 1 : (g > 148 * 16 ? 148 * 16 : g));
}

}  // namespace

void graph_build(const uint8_t *out, const uint64_t *rec_off, const uint64_t *rec_e0, uint32_t nrec, uint64_t E,
                 uint32_t nodes, const GraphBufs &b, cudaStream_t s) {
    const unsigned ge = grid_of(E), gn = grid_of(nodes);
    cudaMemsetAsync(b.dout, 0, (size_t)nodes * 4, s);
    cudaMemsetAsync(b.din, 0, (size_t)nodes * 4, s);
    cudaMemsetAsync(b.succ, 0xff, (size_t)nodes * 4, s);
    cudaMemsetAsync(b.pred, 0xff, (size_t)nodes * 4, s);
    cudaMemsetAsync(b.size, 0, (size_t)nodes * 4, s);
    if (E) {
        count_launch(3);
        graph_scatter_kernel<<<ge, kGT, 0, s>>>(out, rec_off, rec_e0, nrec, E, b.from, b.to);
        graph_degree_kernel<<<ge, kGT, 0, s>>>(b.from, b.to, E, nodes, b.dout, b.din, b.err);
        graph_link_kernel<<<ge, kGT, 0, s>>>(b.from, b.to, E, nodes, b.dout, b.din, b.succ, b.pred);
    }
    int rounds = 1;
    while ((1ull << rounds) < (uint64_t)nodes + 1) ++rounds;
    // the paths from their heads; the nodes left (hop = none) lie on cycles
    cudaMemsetAsync(b.hop[0], 0xff, (size_t)nodes * 4, s);
    graph_walk_kernel<<<gn, kGT, 0, s>>>(b.pred, b.succ, nullptr, nodes, 0, b.hop[0], b.dist[0]);
    // cycle minimum: mn = node, nx = pred, doubling over the cycle nodes only
    launch_iota(b.mn[0], nodes, s);
    cudaMemcpyAsync(b.nx[0], b.pred, (size_t)nodes * 4, cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(b.mn[1], b.mn[0], (size_t)nodes * 4, cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(b.nx[1], b.nx[0], (size_t)nodes * 4, cudaMemcpyDeviceToDevice, s);
    for (int r = 0; r < rounds; ++r)
        graph_cycle_min_kernel<<<gn, kGT, 0, s>>>(b.hop[0], b.mn[r & 1], b.nx[r & 1], nodes, b.mn[(r + 1) & 1],
                                                   b.nx[(r + 1) & 1]);
    graph_cut_kernel<<<gn, kGT, 0, s>>>(b.hop[0], b.mn[rounds & 1], nodes, b.pred, b.succ, b.cycles);
    graph_walk_kernel<<<gn, kGT, 0, s>>>(b.pred, b.succ, b.mn[rounds & 1], nodes, 1, b.hop[0], b.dist[0]);
    count_launch(rounds + 3);
    graph_size_kernel<<<gn, kGT, 0, s>>>(b.hop[0], nodes, b.size);
    launch_scan_u32_u64(b.size, b.start, nodes, b.status, b.tile_ctr, b.total, b.err, s);
    graph_place_kernel<<<gn, kGT, 0, s>>>(b.hop[0], b.dist[0], b.start, nodes, b.order);
    count_launch(2);
}

}  // namespace emp
