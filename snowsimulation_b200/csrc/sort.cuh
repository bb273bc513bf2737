// sort.cuh -- neighbor structure: cell hashing, a stable counting sort of cell hashes,
// and the cell table (cuda_simulation.cu:194-301, :359-420, :1455-1468).
//
// The reference sorts (hash, index) pairs with thrust::sort_by_key, which is stable.
// This is a counting sort over the num_cells cell keys that yields the same
// permutation:
//   1. hash + count: each particle's cell key, and an (unordered) slot in its cell
//      from an atomic counter;
//   2. exclusive scan of the per-cell counts (num_cells + 1 offsets); the same pass
//      re-zeroes the counters and clears cell_start over the range the reference clears;
//   3. scatter each particle into its cell's range (unordered inside the cell);
//   4. rank inside the cell by original index (cells hold a handful of particles),
//      which restores the stable order, then write every output of the reference's
//      reorder pass (grid_hash, grid_index, cell_start/cell_end of occupied cells,
//      sorted_pos) plus the compact float4 copy used by the neighbor loops.
#pragma once
#include "common.cuh"

namespace snowb {

constexpr int SCAN_TPB = 256;                 // threads per scan block
constexpr int SCAN_ITEMS = 4;                 // entries per thread
constexpr int SCAN_CHUNK = SCAN_TPB * SCAN_ITEMS;

__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t v)
{
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    return v;
}
__device__ __forceinline__ uint32_t warp_sum(uint32_t v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block-wide exclusive scan of one value per thread (blockDim.x == SCAN_TPB).
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t* sm, uint32_t& total)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t inc = warp_incl_scan(v);
    if (lane == 31) sm[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < SCAN_TPB / 32 ? sm[lane] : 0u;
        uint32_t wi = warp_incl_scan(w);
        if (lane < SCAN_TPB / 32) sm[lane] = wi - w;
        if (lane == SCAN_TPB / 32 - 1) sm[SCAN_TPB / 32] = wi;
    }
    __syncthreads();
    uint32_t r = sm[warp] + inc - v;
    total = sm[SCAN_TPB / 32];
    __syncthreads();
    return r;
}

// Sum of the first `count` block sums, computed by every thread of warp 0.
__device__ __forceinline__ uint32_t prefix_of_blocks(const uint32_t* bsum, uint32_t count)
{
    uint32_t s = 0;
    for (uint32_t k = threadIdx.x & 31; k < count; k += 32) s += bsum[k];
    return warp_sum(s);
}

// ------------------------------------------------------------------ 1. hash + count
// Fused path: hash of pos[o] for o < n (calcHashD :194-212).  Also adds every particle to
// the count of its scan chunk (bsum, SCAN_CHUNK cells each, one atomic per chunk and warp),
// which the cell scan needs; the scatter pass re-zeroes bsum for the next sort.
// Sort points of a substep decide for themselves (gate.S set): the hash pass turns the
// set's moved flag into the decision (DevState::resort, read by the later passes; the scan
// pass clears the flag), and returns at once when the set keeps its last sort.  The first
// sort point of a substep also opens it (begin).  gate.S null: `cond` alone decides.
struct SortGate {
    DevState* S;
    int set, begin;
};
// substep start: launch sizes, phase-change and link counters
__device__ __forceinline__ void begin_substep(DevState* S)
{
    S->n0_sph = S->n_sph; S->n0_dem = S->n_dem;
    S->n_freeze = 0; S->n_melt = 0; S->changed = 0; S->n_active = 0; S->n_links = 0; S->n_nl_ovf = 0;
    for (int c = 0; c < 8; ++c) S->sc_count[c] = 0u;
}
__global__ void k_hash_count(DevParams P, const snowb_float3* __restrict__ pos, const uint32_t* n_ptr,
                             uint32_t n_fixed, uint32_t* __restrict__ key_o, uint32_t* __restrict__ slot_o,
                             uint32_t* __restrict__ cnt, const uint32_t* cond, const uint32_t* __restrict__ sid_o,
                             uint32_t* __restrict__ bsum, SortGate gate)
{
    if (gate.S) {
        const uint32_t m = gate.S->moved[gate.set];
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            if (gate.begin) begin_substep(gate.S);
            gate.S->resort[gate.set] = m;
            if (m) ++gate.S->sorts_full[gate.set];
            else ++gate.S->sorts_kept[gate.set];
        }
        if (m == 0) return;
    } else if (cond && *cond == 0) return;
    const uint32_t n = n_ptr ? *n_ptr : n_fixed;
    const uint32_t lane = threadIdx.x & 31u;
    // whole warps iterate together so the chunk counts can be aggregated with warp votes
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t base = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < n; base += stride) {
        const uint32_t o = base + lane;
        const bool live = o < n;
        uint32_t chunk = 0xFFFFFFFFu;
        if (live) {
            float3 p = ldv3(pos, o);
            uint32_t h = grid_hash(P, grid_pos(P, p, sid_o ? sid_o[o] : 0u), 0, 0, 0);
            key_o[o] = h;
            slot_o[o] = atomicAdd(cnt + h, 1u);
            chunk = h / (uint32_t)SCAN_CHUNK;
        }
        const uint32_t peers = __match_any_sync(0xffffffffu, chunk);
        if (live && lane == (uint32_t)(__ffs(peers) - 1)) atomicAdd(bsum + chunk, (uint32_t)__popc(peers));
    }
}
// sort_particles path: keys and values already in (grid_hash, grid_index).
__global__ void k_key_count(const uint32_t* __restrict__ keys, const uint32_t* __restrict__ vals, uint32_t n,
                            uint32_t ncells, uint32_t* __restrict__ key_o, uint32_t* __restrict__ val_o,
                            uint32_t* __restrict__ slot_o, uint32_t* __restrict__ cnt, uint32_t* err)
{
    GRID_LOOP(i, n) {
        uint32_t h = keys[i];
        if (h >= ncells) { atomicOr(err, 2u); h = ncells - 1; }
        key_o[i] = h;
        val_o[i] = vals[i];
        slot_o[i] = atomicAdd(cnt + h, 1u);
    }
}

// ------------------------------------------------------------------ 2. scan of counts
__global__ void k_block_sums(const uint32_t* __restrict__ cnt, uint32_t ncells, uint32_t* __restrict__ bsum,
                             const uint32_t* cond)
{
    if (cond && *cond == 0) return;
    __shared__ uint32_t sm[SCAN_TPB / 32];
    const uint32_t base = blockIdx.x * SCAN_CHUNK + threadIdx.x * SCAN_ITEMS;
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k)
        if (base + k < ncells) s += cnt[base + k];
    s = warp_sum(s);
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        uint32_t v = threadIdx.x < SCAN_TPB / 32 ? sm[threadIdx.x] : 0u;
        v = warp_sum(v);
        if (threadIdx.x == 0) bsum[blockIdx.x] = v;
    }
}

// off[c] = exclusive prefix of cnt; off[ncells] = total; cnt re-zeroed; cell_start cleared
// for c < clear (clear = min(n, ncells) reproduces the reference's partial memset, Q1).
// moved: the set's moved flag, cleared here once the hash pass has read it (null: none)
__global__ void k_cell_scan(uint32_t* __restrict__ cnt, const uint32_t* __restrict__ bsum, uint32_t ncells,
                            uint32_t* __restrict__ off, uint32_t* __restrict__ cell_start,
                            const uint32_t* n_ptr, uint32_t n_fixed, int clear_all, const uint32_t* cond,
                            uint32_t* moved = nullptr)
{
    if (moved && blockIdx.x == 0 && threadIdx.x == 0) *moved = 0u;
    if (cond && *cond == 0) return;
    __shared__ uint32_t sm[SCAN_TPB / 32 + 1];
    __shared__ uint32_t s_prefix;
    if (threadIdx.x < 32) {
        uint32_t p = prefix_of_blocks(bsum, blockIdx.x);
        if (threadIdx.x == 0) s_prefix = p;
    }
    const uint32_t n = n_ptr ? *n_ptr : n_fixed;
    const uint32_t clear = clear_all ? ncells : umin32(n, ncells);
    const uint32_t base = blockIdx.x * SCAN_CHUNK + threadIdx.x * SCAN_ITEMS;
    uint32_t v[SCAN_ITEMS], t = 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        v[k] = base + k < ncells ? cnt[base + k] : 0u;
        t += v[k];
    }
    uint32_t total;
    __syncthreads();
    uint32_t ex = block_excl_scan(t, sm, total) + s_prefix;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        uint32_t c = base + k;
        if (c < ncells) {
            off[c] = ex;
            cnt[c] = 0u;
            if (c < clear) cell_start[c] = SNOWB_EMPTY;
            if (c == ncells - 1) off[ncells] = ex + v[k];
        }
        ex += v[k];
    }
}

// ------------------------------------------------------------------ 3. scatter
__global__ void k_scatter(const uint32_t* __restrict__ key_o, const uint32_t* __restrict__ slot_o,
                          const uint32_t* __restrict__ off, uint32_t* __restrict__ tmp,
                          const uint32_t* n_ptr, uint32_t n_fixed, const uint32_t* cond,
                          uint32_t* __restrict__ bsum_zero = nullptr, uint32_t nbsum = 0)
{
    if (cond && *cond == 0) return;
    const uint32_t n = n_ptr ? *n_ptr : n_fixed;
    GRID_LOOP(o, n) tmp[off[key_o[o]] + slot_o[o]] = o;
    if (bsum_zero) GRID_LOOP(k, nbsum) bsum_zero[k] = 0u;
}

// rank of element o among the (unordered) members of its cell, by ascending o
__device__ __forceinline__ uint32_t stable_rank(const uint32_t* __restrict__ tmp, uint32_t b, uint32_t e, uint32_t o)
{
    uint32_t r = 0;
    for (uint32_t k = b; k < e; ++k) r += tmp[k] < o;
    return r;
}

// ------------------------------------------------------------------ 4. rank + outputs
// Fused path (sort_and_reorder :398-420 with hash = cell of pos).  Also gathers the
// compact sorted attributes: p4 = (pos, w[o]), invm_s, contrib_s.  With *cond == 0 the
// sort point keeps the last sort (no particle left its cell, same set size): grid_hash,
// grid_index and the cell table are already what this sort would write, so only the
// gathered outputs are refreshed, sorted slot by sorted slot.
__global__ void k_rank_reorder(const uint32_t* __restrict__ key_o, const uint32_t* __restrict__ off,
                               const uint32_t* __restrict__ tmp, const snowb_float3* __restrict__ pos,
                               const float* __restrict__ w, const float* __restrict__ invm,
                               const float* __restrict__ contrib, snowb_cell_data cd, float4* __restrict__ p4,
                               float* __restrict__ invm_s, float* __restrict__ contrib_s,
                               const uint32_t* n_ptr, uint32_t n_fixed, const uint32_t* cond,
                               const uint32_t* __restrict__ sid_o, uint32_t* __restrict__ sid_s)
{
    const uint32_t n = n_ptr ? *n_ptr : n_fixed;
    if (cond && *cond == 0) {
        GRID_LOOP(p, n) {
            const uint32_t o = cd.grid_index[p];
            const float3 q = ldv3(pos, o);
            st3(cd.sorted_pos, p, q);
            if (p4) p4[p] = make_float4(q.x, q.y, q.z, w ? w[o] : 0.f);
            if (invm_s) invm_s[p] = invm[o];
            if (contrib_s) contrib_s[p] = contrib[o];
            if (sid_s) sid_s[p] = sid_o[o];
        }
        return;
    }
    GRID_LOOP(o, n) {
        const uint32_t h = key_o[o], b = off[h], e = off[h + 1];
        const uint32_t r = stable_rank(tmp, b, e, o);
        const uint32_t p = b + r;
        cd.grid_index[p] = o;
        cd.grid_hash[p] = h;
        if (r == 0) { cd.cell_start[h] = b; cd.cell_end[h] = e; }
        float3 q = ldv3(pos, o);
        st3(cd.sorted_pos, p, q);
        if (p4) p4[p] = make_float4(q.x, q.y, q.z, w ? w[o] : 0.f);
        if (invm_s) invm_s[p] = invm[o];
        if (contrib_s) contrib_s[p] = contrib[o];
        if (sid_s) sid_s[p] = sid_o[o];
    }
}
// A set whose particles all kept their cells since its last sort sorts to the same
// permutation and cell table, so only the gathered outputs change: the kernels that move
// particles compare each new cell with the particle's key at the last sort and mark the
// set when one differs.
struct SortTrack {
    const uint32_t* key;        // cell key per original index at the set's last sort (null: no tracking)
    const uint32_t* sid;        // scene id per original index (batched runs) or null
    uint32_t* moved;            // &DevState::moved[set]
};
__device__ __forceinline__ void track_move(const DevParams& P, const SortTrack& T, uint32_t o, float3 q,
                                           uint32_t scene)
{
    if (grid_hash(P, grid_pos(P, q, scene), 0, 0, 0) != __ldg(T.key + o)) *T.moved = 1u;
}
// sort_particles path: write the sorted keys and values only.
__global__ void k_rank_pairs(const uint32_t* __restrict__ key_o, const uint32_t* __restrict__ val_o,
                             const uint32_t* __restrict__ off, const uint32_t* __restrict__ tmp,
                             uint32_t* __restrict__ keys, uint32_t* __restrict__ vals, uint32_t n)
{
    GRID_LOOP(i, n) {
        const uint32_t h = key_o[i], b = off[h], e = off[h + 1];
        const uint32_t p = b + stable_rank(tmp, b, e, i);
        keys[p] = h;
        vals[p] = val_o[i];
    }
}

// calcHashD (:194-212) alone
__global__ void k_calc_hash(DevParams P, snowb_cell_data cd, const snowb_float3* __restrict__ pos, uint32_t n,
                            const uint32_t* __restrict__ sid_o)
{
    GRID_LOOP(i, n) {
        float3 p = ldv3(pos, i);
        cd.grid_hash[i] = grid_hash(P, grid_pos(P, p, sid_o ? sid_o[i] : 0u), 0, 0, 0);
        cd.grid_index[i] = i;
    }
}
// reorderDataAndFindCellStartD (:242-301) alone; cell_start cleared beforehand
__global__ void k_reorder(snowb_cell_data cd, const snowb_float3* __restrict__ pos, uint32_t n)
{
    GRID_LOOP(i, n) {
        const uint32_t h = cd.grid_hash[i];
        if (i == 0 || h != cd.grid_hash[i - 1]) {
            cd.cell_start[h] = i;
            if (i > 0) cd.cell_end[cd.grid_hash[i - 1]] = i;
        }
        if (i == n - 1) cd.cell_end[h] = i + 1;
        st3(cd.sorted_pos, i, ldv3(pos, cd.grid_index[i]));
    }
}
// Occupied ranges of a sorted hash array (fresh, without stale entries); the tables are
// zeroed beforehand so empty cells read [0, 0).
__global__ void k_fresh_ranges(const uint32_t* __restrict__ hash, uint32_t n, uint32_t* __restrict__ fs,
                               uint32_t* __restrict__ fe)
{
    GRID_LOOP(i, n) {
        const uint32_t h = hash[i];
        if (i == 0 || hash[i - 1] != h) fs[h] = i;
        if (i == n - 1 || hash[i + 1] != h) fe[h] = i + 1;
    }
}

// ------------------------------------------------------------------ generic scan
// Exclusive scan of in[0, n) into out (n from device or fixed), total into *total.
__global__ void k_scan_sums(const uint32_t* __restrict__ in, const uint32_t* n_ptr, uint32_t n_fixed,
                            uint32_t* __restrict__ bsum, const uint32_t* cond)
{
    if (cond && *cond == 0) return;
    const uint32_t n = n_ptr ? *n_ptr : n_fixed;
    __shared__ uint32_t sm[SCAN_TPB / 32];
    const uint32_t base = blockIdx.x * SCAN_CHUNK + threadIdx.x * SCAN_ITEMS;
    if (blockIdx.x * SCAN_CHUNK >= n && blockIdx.x != 0) { if (threadIdx.x == 0) bsum[blockIdx.x] = 0; return; }
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k)
        if (base + k < n) s += in[base + k];
    s = warp_sum(s);
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        uint32_t v = threadIdx.x < SCAN_TPB / 32 ? sm[threadIdx.x] : 0u;
        v = warp_sum(v);
        if (threadIdx.x == 0) bsum[blockIdx.x] = v;
    }
}
__global__ void k_scan_apply(const uint32_t* __restrict__ in, const uint32_t* n_ptr, uint32_t n_fixed,
                             const uint32_t* __restrict__ bsum, uint32_t* __restrict__ out, uint32_t* total,
                             const uint32_t* cond)
{
    if (cond && *cond == 0) return;
    const uint32_t n = n_ptr ? *n_ptr : n_fixed;
    const uint32_t nblocks = (n + SCAN_CHUNK - 1) / SCAN_CHUNK;
    if (n == 0) { if (blockIdx.x == 0 && threadIdx.x == 0 && total) *total = 0; return; }
    if (blockIdx.x >= nblocks) return;
    __shared__ uint32_t sm[SCAN_TPB / 32 + 1];
    __shared__ uint32_t s_prefix;
    if (threadIdx.x < 32) {
        uint32_t p = prefix_of_blocks(bsum, blockIdx.x);
        if (threadIdx.x == 0) s_prefix = p;
    }
    const uint32_t base = blockIdx.x * SCAN_CHUNK + threadIdx.x * SCAN_ITEMS;
    uint32_t v[SCAN_ITEMS], t = 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        v[k] = base + k < n ? in[base + k] : 0u;
        t += v[k];
    }
    uint32_t tot;
    __syncthreads();
    uint32_t ex = block_excl_scan(t, sm, tot) + s_prefix;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        if (base + k < n) {
            if (out) out[base + k] = ex;
            if (base + k == n - 1 && total) *total = ex + v[k];
        }
        ex += v[k];
    }
}

}  // namespace snowb
