// phase.cuh -- freezing/melting with compaction (cuda_simulation.cu:3974-4125, :4387-4622)
// and interlink formation (:4127-4292, :4768-4816).
//
// Phase change.  The reference claims target slots with atomicAdd, so their order is
// scheduling dependent (Q8); here a particle's target is its rank among the particles
// changing phase (ascending index).  Compaction always runs in the reference; when no
// particle changed phase it is an identity, so every compaction kernel returns early
// unless DevState::changed is set (no host round trip is needed).
//
// Interlink formation.  The reference lets every snow particle claim slots with atomics
// while others read the same slots (Q10), so the topology depends on scheduling.  Here
// the pass is the sequential reference procedure applied in one fixed order: hash cells
// are grouped into 2x2x2 super-cells, each super-cell gets a colour 0..7 from the parity
// of its coordinates, colours run in turn, and inside a colour each super-cell walks its
// particles in ascending sorted index.  A particle only edits its own slots and those of
// neighbours within h, i.e. in adjacent cells; same-coloured super-cells are at least
// three cells apart, so they never touch the same particle and run in parallel, one
// thread per super-cell.  A prefilter marks the particles that can change anything:
// links are never removed during the pass and counts only grow, so a particle whose
// count already reaches its cap, or whose candidates are all linked already, is a no-op.
#pragma once
#include "common.cuh"
#include "sort.cuh"

namespace snowb {

#define SNOWB_MAXC_FAST 32   // interlink slots kept in registers (maximum_connection <= 32)

// copy_particle_info (:3974-4002): every per-particle field, then the link slots
__device__ __forceinline__ void copy_fields(const snowb_particle_data& s, const snowb_particle_data& d, uint32_t i,
                                            uint32_t t)
{
    st3(d.positions, t, ldv3(s.positions, i));
    st3(d.predict_positions, t, ldv3(s.predict_positions, i));
    st3(d.new_positions, t, ldv3(s.new_positions, i));
    st3(d.velocity, t, ldv3(s.velocity, i));
    st3(d.force, t, ldv3(s.force, i));
    st3(d.correction, t, ldv3(s.correction, i));
    d.mass[t] = s.mass[i];
    d.massInv[t] = s.massInv[i];
    d.contrib[t] = s.contrib[i];
    d.density[t] = s.density[i];
    d.C[t] = s.C[i];
    d.lambda[t] = s.lambda[i];
    d.T[t] = s.T[i];
    d.new_T[t] = s.new_T[i];
    d.trackId[t] = s.trackId[i];
    d.iter_end[t] = s.iter_end[i];
}
__device__ __forceinline__ void copy_info(const snowb_particle_data& s, const snowb_particle_data& d, uint32_t i,
                                          uint32_t t, uint32_t M)
{
    copy_fields(s, d, i, t);
    for (uint32_t c = 0; c < M; ++c) {
        d.connect_record[t * M + c] = s.connect_record[i * M + c];
        d.connect_length[t * M + c] = s.connect_length[i * M + c];
    }
}
__device__ __forceinline__ void reset_records(const snowb_particle_data& d, uint32_t t, uint32_t M)
{
    for (uint32_t c = 0; c < M; ++c) {
        d.connect_record[t * M + c] = SNOWB_UMAX;
        d.connect_length[t * M + c] = 0.f;
    }
    d.iter_end[t] = M * t;
}

// freeze / melt predicates (:4425, :4396)
// commit: the heat pass's commit (k_heat_commit: T from new_T, plus the environment
// term) first, each particle its own, so the flags read the committed temperature
__global__ void k_phase_flags(DevParams P, const DevState* __restrict__ S, snowb_particle_data sph,
                              snowb_particle_data dem, int freeze, int melt, uint32_t* __restrict__ fl_s,
                              uint32_t* __restrict__ fl_d, int commit, float dTe, int env_sph, int env_dem)
{
    const uint32_t ns = S->n_sph, nd = S->n_dem;
    GRID_LOOP(t, ns + nd) {
        const bool w = t < ns;
        const uint32_t i = w ? t : t - ns;
        const snowb_particle_data& D = w ? sph : dem;
        float T;
        if (commit) {
            T = D.new_T[i];
            if (w ? env_sph : env_dem) T += dTe;
            D.T[i] = T;
        } else {
            T = D.T[i];
        }
        if (w) fl_s[i] = (freeze && T <= P.Tf && sph.contrib[i] >= 0.99f) ? 1u : 0u;
        else fl_d[i] = (melt && T > P.Tf && dem.contrib[i] >= 0.99f) ? 1u : 0u;
    }
}
// scene ids of batched runs travel with the particles (null pointers: one scene)
struct SceneIds {
    uint32_t *sph, *dem, *buf;
};
// freezing (:4416-4449) and melting (:4387-4414) with ranked targets, and the phase-change
// flag: every block derives it from the counts, block 0 stores it for the later passes
__global__ void k_phase_move(DevParams P, DevState* __restrict__ S, snowb_particle_data sph,
                             snowb_particle_data dem, const uint32_t* __restrict__ fl_s,
                             const uint32_t* __restrict__ rk_s, const uint32_t* __restrict__ fl_d,
                             const uint32_t* __restrict__ rk_d, SceneIds sc)
{
    const bool changed = (S->n_freeze + S->n_melt) != 0u;
    if (blockIdx.x == 0 && threadIdx.x == 0) S->changed = changed ? 1u : 0u;
    if (!changed) return;
    const uint32_t ns = S->n_sph, nd = S->n_dem, M = P.maxc;
    GRID_LOOP(t, ns + nd) {
        if (t < ns) {
            if (!fl_s[t]) continue;
            const uint32_t i = t, tg = nd + rk_s[i];
            sph.contrib[i] = 0.f;
            copy_info(sph, dem, i, tg, M);
            if (sc.sph) sc.dem[tg] = sc.sph[i];
            sph.predicate[i] = 0; sph.trackId[i] = 0;
            dem.predicate[tg] = 1;
            reset_records(dem, tg, M);
        } else {
            const uint32_t i = t - ns;
            if (!fl_d[i]) continue;
            const uint32_t tg = ns + rk_d[i];
            dem.contrib[i] = 0.f;
            copy_info(dem, sph, i, tg, M);
            if (sc.sph) sc.sph[tg] = sc.dem[i];
            dem.predicate[i] = 0; dem.trackId[i] = 0;
            sph.predicate[tg] = 1;
        }
    }
}
// Compaction moves the kept particles to their ranks (scan_index).  A kept particle with
// no removed one before it stays where it is, and copying it out and back, as the
// reference's copy_to_target and scatter do for every slot, leaves it unchanged; so both
// passes move only the particles whose slot changes (the phase-change buffer, scratch the
// reference overwrites at every compaction, holds only those).  Threads k < full take a
// particle's fields, the others one link slot each (coalesced over the slot arrays).
__device__ __forceinline__ bool compaction_moves(const snowb_particle_data& d, uint32_t i)
{
    return d.predicate[i] == 1 && d.scan_index[i] != i;
}
// copy_to_target (:4451-4460) into the caller's phase-change buffer.  removed: the
// number of particles the set loses (none: no particle moves)
__global__ void k_copy_to_buffer(DevParams P, const DevState* __restrict__ S, snowb_particle_data d,
                                 snowb_particle_data buf, uint32_t full, const uint32_t* __restrict__ sid,
                                 uint32_t* __restrict__ sid_buf, const uint32_t* __restrict__ removed)
{
    if (S->changed == 0 || *removed == 0) return;
    const uint32_t M = P.maxc;
    GRID_LOOP(k, full * (M + 1)) {
        if (k < full) {
            if (!compaction_moves(d, k)) continue;
            copy_fields(d, buf, k, k);
            if (sid) sid_buf[k] = sid[k];
        } else {
            const uint32_t s = k - full;
            if (!compaction_moves(d, s / M)) continue;
            buf.connect_record[s] = d.connect_record[s];
            buf.connect_length[s] = d.connect_length[s];
        }
    }
}
// scatter (:4462-4480).  rebase (fixed quirks, snow set): a moved particle keeps its link
// count, iter_end = t*M + count; the reference copies iter_end verbatim (Q13).  A particle
// that stays keeps its iter_end either way.
__global__ void k_scatter_set(DevParams P, DevState* S, snowb_particle_data d, snowb_particle_data buf, uint32_t full,
                              uint32_t* __restrict__ sid, const uint32_t* __restrict__ sid_buf, int rebase,
                              const uint32_t* __restrict__ removed)
{
    if (S->changed == 0) return;
    const uint32_t M = P.maxc;
    // with nothing removed every kept particle stays: only new_index is written
    GRID_LOOP(k, *removed ? full * (M + 1) : full) {
        if (k < full) {
            const uint32_t i = k;
            if (d.predicate[i] == 1) {
                const uint32_t t = d.scan_index[i];
                if (t >= full) { atomicOr(&S->err, SNOWB_DEVERR_SCATTER); continue; }
                if (t != i) {
                    copy_fields(buf, d, i, t);
                    if (rebase) d.iter_end[t] = M * t + (buf.iter_end[i] - M * i);
                    if (sid) sid[t] = sid_buf[i];
                }
                d.new_index[i] = t;
            } else d.new_index[i] = SNOWB_UMAX;
        } else {
            const uint32_t s = k - full, i = s / M;
            if (d.predicate[i] != 1) continue;
            const uint32_t t = d.scan_index[i];
            if (t >= full || t == i) continue;
            const uint32_t q = t * M + (s - i * M);
            d.connect_record[q] = buf.connect_record[s];
            d.connect_length[q] = buf.connect_length[s];
        }
    }
}
// setSize / new_end (:4545-4551), predicate fill (:4555-4556), clean_tail (:4482-4493).
// The reference compacts every substep; without a phase change that is an identity except
// that it zeroes scan_index in the tail and, if a link pass wrote into tail slots, resets
// them (`full_clean`), which is what this kernel does in that case.
// The tail clean only has to reach the slots that can differ from a clean slot: those that
// held a particle before this compaction (below the set's size plus the particles it
// gained) and those not known clean since the last clean (DevState::clean_hi; a call's
// first compaction and any link pass that wrote past a set's end, tail_dirty, clean the
// whole tail).  A slot at or above both already holds what the clean writes.
// records: also the record update below (update_record_index; its slots, below the new
// snow size, are none of the tail slots this pass cleans), in the same launch
__device__ __forceinline__ void update_record(const DevParams& P, const DevState* S, const snowb_particle_data& dem,
                                              uint32_t s, bool moved, uint32_t nd_old, uint32_t nd);
__global__ void k_compact_finish(DevParams P, DevState* S, snowb_particle_data sph, snowb_particle_data dem,
                                 uint32_t full, int records)
{
    const bool full_clean = S->changed || S->tail_dirty;
    const uint32_t sn = S->new_sph, dn = S->new_dem, M = P.maxc;
    const uint32_t hs = S->tail_dirty ? full : umin32(full, umax32(S->clean_hi[0], S->n_sph + S->n_melt));
    const uint32_t hd = S->tail_dirty ? full : umin32(full, umax32(S->clean_hi[1], S->n_dem + S->n_freeze));
    const bool moved = S->changed != 0;
    const uint32_t nd_old = S->n_dem, nd_rec = moved ? S->new_dem : S->n_dem;
    const uint32_t nrec = records && full_clean ? M * nd_rec : 0u;
    GRID_LOOP(t, 2 * full + nrec) {
        if (t >= 2 * full) {
            update_record(P, S, dem, t - 2 * full, moved, nd_old, nd_rec);
            continue;
        }
        const bool w = t < full;
        const uint32_t i = w ? t : t - full;
        const snowb_particle_data& d = w ? sph : dem;
        const uint32_t n = w ? sn : dn;
        if (i < n) {
            if (full_clean) d.predicate[i] = 1;
        } else {
            d.scan_index[i] = 0;
            if (full_clean && i < (w ? hs : hd)) {
                d.predicate[i] = 0; d.trackId[i] = 0;
                reset_records(d, i, M);
            }
        }
        if (i == 0 && full_clean) *d.new_end = n;
    }
}
// The compaction's last launch: the new sizes (a compacted set is sorted in full next),
// the clean mark of the tails, and the tail flag cleared.
__global__ void k_commit_sizes(DevState* S)
{
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        // after a clean every slot past the new sizes is clean
        if (S->changed || S->tail_dirty) { S->clean_hi[0] = S->new_sph; S->clean_hi[1] = S->new_dem; }
        if (S->changed) {
            S->n_sph = S->new_sph; S->n_dem = S->new_dem;
            S->moved[0] = 1u; S->moved[1] = 1u;
        }
        S->tail_dirty = 0;
    }
}
// update_record_index (:4114-4125), after the compaction, with shuffle_useless_record
// (:4068-4111) folded in: the reference clears, before the compaction, each link to a
// partner that left the snow set (its record, its length, one off the owner's count).  The
// link's slot moves with its owner and the partner's new index is then empty, so the same
// slot is cleared here at the owner's new place; the count's decrement commutes with the
// compaction's copy or rebase of it.
__device__ __forceinline__ void update_record(const DevParams& P, const DevState* S, const snowb_particle_data& dem,
                                              uint32_t s, bool moved, uint32_t nd_old, uint32_t nd)
{
    const uint32_t r = dem.connect_record[s];
    if (r == SNOWB_UMAX) return;
    if (moved) {
        const uint32_t nr = dem.new_index[r];
        if (r < nd_old && nr == SNOWB_UMAX) {
            dem.connect_length[s] = 0.f;
            atomicSub(dem.iter_end + s / P.maxc, 1u);
        }
        dem.connect_record[s] = nr;
    } else {
        // without a phase change the reference's new_index is the identity below n, empty above
        dem.connect_record[s] = r < nd ? r : SNOWB_UMAX;
    }
}

// ======================================================================= links
__device__ __forceinline__ uint32_t link_tolerance(const DevParams& P, float T, int dynamic)
{
    uint32_t tol = dynamic ? __float2uint_rz(((T - P.Tf) / (P.Th - P.Tf)) * (float)P.maxc) : P.maxc;
    return tol < P.maxc ? tol : P.maxc;
}
// Prefilter: can particle (sorted) i change any record in this pass?  During the pass
// links are only added and counts only grow, so i is a no-op if its count already reaches
// its cap, if it has no free slot, or if every candidate (d < h) is either linked to it
// already or has no room (count at the cap or no free slot): an attempt on a full
// partner claims a slot of i and releases it again.  A candidate that is i itself (a
// stale cell range can hold it) keeps i active.
__device__ __forceinline__ bool has_free_slot(const uint32_t* rec, uint32_t o, uint32_t M)
{
    for (uint32_t q = M * o; q < M * (o + 1); ++q)
        if (rec[q] == SNOWB_UMAX) return true;
    return false;
}
// Super-cells holding an active particle, listed per colour by the prefilter so that a
// colour pass visits only those (same-coloured super-cells are independent, so their order
// does not matter; inside one the particles are still taken in ascending sorted index).
// flag null: no list, the colour pass visits every super-cell of its colour.
struct SCList {
    uint32_t* flag;     // per super-cell (colour c, index t at c * per + t): listed
    uint32_t* list;     // colour c's listed indices t at list[c * per + k], k < count[c]
    uint32_t* count;    // DevState::sc_count
    uint32_t per;       // super-cells per colour
};
// colour and index within the colour of the super-cell holding hash cell h (the layout of
// k_link_colour_warp: super-cell (sx, sy, sz) = cell / 2, colour = parities of sx, sy, sz)
__device__ __forceinline__ void supercell_of(const DevParams& P, uint32_t h, uint32_t& colour, uint32_t& t)
{
    const uint32_t x = h % P.gsx, y = (h / P.gsx) % P.gsy, z = h / (P.gsx * P.gsy);
    const uint32_t sx = x >> 1, sy = y >> 1, sz = z >> 1;
    colour = (sx & 1u) | ((sy & 1u) << 1) | ((sz & 1u) << 2);
    t = (sx >> 1) + (P.gsx >> 2) * ((sy >> 1) + (P.gsy >> 2) * (sz >> 1));
}
__device__ __forceinline__ void list_supercell(const DevParams& P, const SCList& sc, uint32_t h)
{
    uint32_t colour, t;
    supercell_of(P, h, colour, t);
    if (atomicCAS(sc.flag + colour * sc.per + t, 0u, 1u) == 0u)
        sc.list[colour * sc.per + atomicAdd(sc.count + colour, 1u)] = t;
}

// L: the snow-snow candidate lists of the substep's first density pass (L.cnt null: none),
// replayed instead of the traversal while no phase change re-sorted the sets.
constexpr uint32_t LF_G = 4;
__global__ void __launch_bounds__(256) k_link_filter(DevParams P, DevState* S, SetView vd,
                                                     snowb_particle_data dem, int dynamic,
                                                     uint8_t* __restrict__ active, NList L, SCList sc)
{
    const uint32_t nd = S->n_dem, M = P.maxc;
    vd.n = nd;
    const bool lists = L.cnt != nullptr && S->changed == 0;
    GRID_LOOP(i, nd) {
        const uint32_t o = vd.gi[i];
        const float3 p = vd.pos(i);
        const uint32_t count = dem.iter_end[o] - o * M;
        uint8_t act = 0;
        // With dynamic caps, adjust_connections (:4768-4808) can leave iter_end below the
        // particle's first slot (it decrements for every slot past the cap, empty ones
        // included), so count wraps round; links that partners add during the pass then
        // bring it back below the cap.  Such a particle is kept: the pass decides.
        if (dem.iter_end[o] < o * M) {
            active[i] = 1;
            atomicAdd(&S->n_active, 1u);
            if (sc.flag) list_supercell(P, sc, vd.gh[i]);
            continue;
        }
        // a particle at its cap stays inactive: its slots are not even read
        const bool below = count < link_tolerance(P, dem.T[o], dynamic);
        // own slots in registers (M <= SNOWB_MAXC_FAST), else read from memory
        uint32_t r[SNOWB_MAXC_FAST];
        const bool fast = M <= SNOWB_MAXC_FAST;
#pragma unroll
        for (int k = 0; k < SNOWB_MAXC_FAST; ++k)
            r[k] = below && fast && (uint32_t)k < M ? dem.connect_record[M * o + k] : 0u;
        const uint32_t lc = lists ? L.cnt[L.cap + i] : NL_OVF;
        // a free slot of o: from the registers (slots k >= M hold 0, never empty)
        bool own_free = false;
        if (below) {
            if (fast) {
#pragma unroll
                for (int k = 0; k < SNOWB_MAXC_FAST; ++k) own_free |= r[k] == SNOWB_UMAX;
            } else {
                own_free = has_free_slot(dem.connect_record, o, M);
            }
        }
        if (!(lc & NL_OVF) && own_free) {
            // the same scan over the listed candidates (cells in order, d < h, j != i), taken
            // LF_G at a time: entries, partners' original indices and counts are loaded for
            // the group (all in range: listed entries are current sorted indices), then the
            // candidates are examined in order
            uint32_t skip_cell = 0xFFu;
            const uint32_t nl = lc & 1023u;
            for (uint32_t k0 = 0; k0 < nl && !act; k0 += LF_G) {
                uint32_t en[LF_G], o1[LF_G], ie[LF_G];
#pragma unroll
                for (uint32_t u = 0; u < LF_G; ++u)
                    en[u] = k0 + u < nl ? L.e[(size_t)(k0 + u) * L.stride + L.cap + i] : 0u;
#pragma unroll
                for (uint32_t u = 0; u < LF_G; ++u) o1[u] = k0 + u < nl ? vd.gi[en[u] & NL_J_MASK] : 0u;
#pragma unroll
                for (uint32_t u = 0; u < LF_G; ++u) ie[u] = k0 + u < nl ? dem.iter_end[o1[u]] : 0u;
#pragma unroll
                for (uint32_t u = 0; u < LF_G; ++u) {
                    if (k0 + u >= nl || act) break;
                    const uint32_t cell = (en[u] >> 25) & 31u;
                    if (cell == skip_cell) continue;
                    if (o1[u] == o) { act = 1; break; }
                    bool found = false;
                    if (fast) {
#pragma unroll
                        for (int q = 0; q < SNOWB_MAXC_FAST; ++q) found |= (uint32_t)q < M && r[q] == o1[u];
                    } else {
                        for (uint32_t q = M * o; q < M * (o + 1); ++q)
                            if (dem.connect_record[q] == o1[u]) { found = true; break; }
                    }
                    if (found) { skip_cell = cell; continue; }
                    if (ie[u] < (o1[u] + 1) * M && has_free_slot(dem.connect_record, o1[u], M)) act = 1;
                }
            }
        } else if ((lc & NL_OVF) && own_free) {
            const GCell g = grid_pos(P, p, vd.scene(i));
            FOR27 {
                uint32_t s, e;
                if (!vd.range(P, g, ox, oy, oz, s, e)) continue;
                for (uint32_t j = s; j < e && !act; ++j) {
                    if (j == i) continue;
                    float3 dv = sub3(p, vd.pos(j));
                    if (dot3(dv, dv) < P.h2_lt) {
                        const uint32_t o1 = vd.gi[j];
                        if (o1 == o) { act = 1; break; }
                        bool found = false;
                        if (fast) {
#pragma unroll
                            for (int k = 0; k < SNOWB_MAXC_FAST; ++k) found |= (uint32_t)k < M && r[k] == o1;
                        } else {
                            for (uint32_t q = M * o; q < M * (o + 1); ++q)
                                if (dem.connect_record[q] == o1) { found = true; break; }
                        }
                        // a linked candidate ends the reference's scan of this cell, and it
                        // stays linked, so nothing after it in the cell is reached
                        if (found) break;
                        if (dem.iter_end[o1] < (o1 + 1) * M && has_free_slot(dem.connect_record, o1, M)) act = 1;
                    }
                }
                if (act) break;
            }
        }
        active[i] = act;
        if (act) {
            atomicAdd(&S->n_active, 1u);
            if (sc.flag) list_supercell(P, sc, vd.gh[i]);
        }
    }
}
// connect_and_record_cell (:4127-4252) + connect_and_record_d (:4255-4284) for one particle.
// Only this thread edits particle o and its neighbours during the colour phase, so o's
// slots, count and tolerance are kept in registers (M <= SNOWB_MAXC_FAST); every record
// write goes through to memory, where the partner search reads it.  Candidates are
// screened with the exact squared-distance test (dist < h <=> d2 < h2_lt).
__device__ void link_particle_fast(const DevParams& P, const SetView& vd, const snowb_particle_data& d, uint32_t i,
                                   int dynamic, DevState* S)
{
    const uint32_t M = P.maxc;
    const float3 p = vd.pos(i);
    const uint32_t o = vd.gi[i];
    const GCell g = grid_pos(P, p, vd.scene(i));
    const uint32_t tol = link_tolerance(P, d.T[o], dynamic);
    const uint32_t base = o * M;
    uint32_t count = d.iter_end[o] - base;
    uint32_t r[SNOWB_MAXC_FAST];
#pragma unroll
    for (int k = 0; k < SNOWB_MAXC_FAST; ++k) r[k] = (uint32_t)k < M ? d.connect_record[base + k] : 0u;
    FOR27 {
        uint32_t s, e;
        if (!vd.range(P, g, ox, oy, oz, s, e)) continue;
        for (uint32_t j = s; j < e; ++j) {
            if (j == i) continue;
            const float3 dv = sub3(p, vd.pos(j));
            const float d2 = dot3(dv, dv);
            if (!(d2 < P.h2_lt) || !(count < tol)) continue;
            const uint32_t o1 = vd.gi[j];
            const float dist = sqrtf(d2);
            bool dup = false;
            int free_k = -1;
#pragma unroll
            for (int k = 0; k < SNOWB_MAXC_FAST; ++k) {
                if ((uint32_t)k < M) {
                    dup |= r[k] == o1;
                    if (free_k < 0 && r[k] == SNOWB_UMAX) free_k = k;
                }
            }
            if (dup) break;               // the reference returns from the cell helper
            if (free_k < 0) continue;     // no free slot: the claim loop finds nothing
            d.connect_record[base + free_k] = o1;           // claim
            bool valid = false;
            const uint32_t b1 = o1 * M;
            if (d.iter_end[o1] < b1 + M)
                for (uint32_t q = b1; q < b1 + M; ++q)
                    if (d.connect_record[q] == SNOWB_UMAX) {
                        d.connect_record[q] = o;
                        d.connect_length[q] = dist;
                        d.iter_end[o1]++;
                        if (o1 >= vd.n) atomicOr(&S->tail_dirty, 1u);
                        if (o1 == o) {                       // self link (stale cell range)
                            ++count;
#pragma unroll
                            for (int k = 0; k < SNOWB_MAXC_FAST; ++k)
                                if ((uint32_t)k == q - base) r[k] = o;
                        }
                        valid = true;
                        break;
                    }
            if (valid) {
                d.connect_length[base + free_k] = dist;
                ++count;
                d.iter_end[o] = base + count;
#pragma unroll
                for (int k = 0; k < SNOWB_MAXC_FAST; ++k)
                    if (k == free_k) r[k] = o1;
                atomicAdd(&S->n_links, 1u);
            } else {
                d.connect_record[base + free_k] = SNOWB_UMAX;
            }
        }
    }
}
// link_particle_fast with the candidate scan spread over a warp.  The warp walks the 27
// cells in order; in each cell 32 candidates at a time are tested for d < h in parallel
// and the passing ones are handled one after another in ascending index, by the same
// sequential rule as link_particle_fast (the dup test ends the cell, own slots are kept in
// registers, claims go through memory).  Every lane holds the same state; lane 0 writes.
// Results are those of link_particle_fast.
__device__ void link_particle_warp(const DevParams& P, const SetView& vd, const snowb_particle_data& d, uint32_t i,
                                   int dynamic, DevState* S)
{
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t M = P.maxc;
    const float3 p = vd.pos(i);
    const uint32_t o = vd.gi[i];
    const GCell g = grid_pos(P, p, vd.scene(i));
    const uint32_t tol = link_tolerance(P, d.T[o], dynamic);
    const uint32_t base = o * M;
    uint32_t count = d.iter_end[o] - base;
    // own slots: lane k holds slot k
    uint32_t rk = lane < M ? d.connect_record[base + lane] : 0u;
    FOR27 {
        uint32_t s, e;
        if (!vd.range(P, g, ox, oy, oz, s, e)) continue;
        bool cell_done = false;
        for (uint32_t j0 = s; j0 < e && !cell_done; j0 += 32u) {
            const uint32_t j = j0 + lane;
            float d2 = 0.f;
            bool in = false;
            if (j < e && j != i) {
                const float3 dv = sub3(p, vd.pos(j));
                d2 = dot3(dv, dv);
                in = d2 < P.h2_lt;
            }
            uint32_t mask = __ballot_sync(0xffffffffu, in);
            while (mask) {
                const int k = __ffs(mask) - 1;
                mask &= mask - 1u;
                if (!(count < tol)) continue;
                const uint32_t jj = j0 + (uint32_t)k;
                const float dk2 = __shfl_sync(0xffffffffu, d2, k);
                const uint32_t o1 = vd.gi[jj];
                const float dist = sqrtf(dk2);
                const bool dup = __any_sync(0xffffffffu, lane < M && rk == o1);
                if (dup) { cell_done = true; break; }   // the reference returns from the cell helper
                const uint32_t freem = __ballot_sync(0xffffffffu, lane < M && rk == SNOWB_UMAX);
                if (!freem) continue;                      // no free slot: the claim loop finds nothing
                const int free_k = __ffs(freem) - 1;
                if (lane == 0) d.connect_record[base + free_k] = o1;   // claim
                if (lane == (uint32_t)free_k) rk = o1;
                __syncwarp();
                const uint32_t b1 = o1 * M;
                bool valid = false;
                if (d.iter_end[o1] < b1 + M) {
                    const uint32_t q = lane < M ? d.connect_record[b1 + lane] : 0u;
                    const uint32_t pm = __ballot_sync(0xffffffffu, lane < M && q == SNOWB_UMAX);
                    if (pm) {
                        const int pk = __ffs(pm) - 1;
                        if (lane == 0) {
                            d.connect_record[b1 + pk] = o;
                            d.connect_length[b1 + pk] = dist;
                            d.iter_end[o1]++;
                            if (o1 >= vd.n) atomicOr(&S->tail_dirty, 1u);
                        }
                        if (o1 == o) {                       // self link (stale cell range)
                            ++count;
                            if (lane == (uint32_t)pk) rk = o;
                        }
                        valid = true;
                    }
                }
                if (valid) {
                    ++count;
                    if (lane == 0) {
                        d.connect_length[base + free_k] = dist;
                        d.iter_end[o] = base + count;
                        atomicAdd(&S->n_links, 1u);
                    }
                } else {
                    if (lane == 0) d.connect_record[base + free_k] = SNOWB_UMAX;
                    if (lane == (uint32_t)free_k) rk = SNOWB_UMAX;
                }
                __syncwarp();
            }
        }
    }
}
// link_particle_warp replaying the snow-snow candidate list written by the substep's first
// density pass at the same sorted positions (entries in traversal order: cells z-y-x, index
// ascending, all with d < h, tagged with their cell).  The sequential rule is the same; a
// dup ends the entries of its cell.
__device__ void link_particle_list(const DevParams& P, const SetView& vd, const snowb_particle_data& d, uint32_t i,
                                   int dynamic, DevState* S, const NList& L, uint32_t n_list)
{
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t M = P.maxc;
    const float3 p = vd.pos(i);
    const uint32_t o = vd.gi[i];
    const uint32_t tol = link_tolerance(P, d.T[o], dynamic);
    const uint32_t base = o * M;
    const uint32_t slot = L.cap + i;
    uint32_t count = d.iter_end[o] - base;
    uint32_t rk = lane < M ? d.connect_record[base + lane] : 0u;
    uint32_t skip_cell = 0xFFu;
    for (uint32_t k0 = 0; k0 < n_list; k0 += 32u) {
        const uint32_t k = k0 + lane;
        uint32_t j = 0, cell = 0xFEu, og = 0;
        float d2 = 0.f;
        if (k < n_list) {
            const uint32_t en = L.e[(size_t)k * L.stride + slot];
            j = en & NL_J_MASK;
            cell = (en >> 25) & 31u;
            const float3 dv = sub3(p, vd.pos(j));
            d2 = dot3(dv, dv);
            // the partner's index, fetched side by side for the 32 candidates (it never
            // changes in this pass), so the walk below needs no load for a duplicate
            og = vd.gi[j];
        }
        // Candidates of a cell are contiguous and in order.  Once a cell is skipped (a
        // duplicate ends it, as the reference returns from its cell helper), its remaining
        // candidates leave the mask in one step; once the count reaches the cap, no later
        // candidate can do anything (counts only grow), so the walk ends.
        if (!(count < tol)) break;
        uint32_t mask = __ballot_sync(0xffffffffu, k < n_list && cell != skip_cell);
        while (mask) {
            const int kk = __ffs(mask) - 1;
            mask &= mask - 1u;
            const uint32_t ck = __shfl_sync(0xffffffffu, cell, kk);
            if (!(count < tol)) break;
            const uint32_t o1 = __shfl_sync(0xffffffffu, og, kk);
            const bool dup = __any_sync(0xffffffffu, lane < M && rk == o1);
            if (dup) {
                skip_cell = ck;
                mask &= ~__ballot_sync(0xffffffffu, cell == ck);
                continue;
            }
            const float dist = sqrtf(__shfl_sync(0xffffffffu, d2, kk));
            const uint32_t freem = __ballot_sync(0xffffffffu, lane < M && rk == SNOWB_UMAX);
            if (!freem) continue;
            const int free_k = __ffs(freem) - 1;
            if (lane == 0) d.connect_record[base + free_k] = o1;
            if (lane == (uint32_t)free_k) rk = o1;
            __syncwarp();
            const uint32_t b1 = o1 * M;
            bool valid = false;
            if (d.iter_end[o1] < b1 + M) {
                const uint32_t q = lane < M ? d.connect_record[b1 + lane] : 0u;
                const uint32_t pm = __ballot_sync(0xffffffffu, lane < M && q == SNOWB_UMAX);
                if (pm) {
                    const int pk = __ffs(pm) - 1;
                    if (lane == 0) {
                        d.connect_record[b1 + pk] = o;
                        d.connect_length[b1 + pk] = dist;
                        d.iter_end[o1]++;
                        if (o1 >= vd.n) atomicOr(&S->tail_dirty, 1u);
                    }
                    if (o1 == o) {
                        ++count;
                        if (lane == (uint32_t)pk) rk = o;
                    }
                    valid = true;
                }
            }
            if (valid) {
                ++count;
                if (lane == 0) {
                    d.connect_length[base + free_k] = dist;
                    d.iter_end[o] = base + count;
                    atomicAdd(&S->n_links, 1u);
                }
            } else {
                if (lane == 0) d.connect_record[base + free_k] = SNOWB_UMAX;
                if (lane == (uint32_t)free_k) rk = SNOWB_UMAX;
            }
            __syncwarp();
        }
    }
}
// One colour with one warp per super-cell: the warp walks the super-cell's particles in
// ascending sorted index and links the active ones with link_particle_warp.
// L: the snow-snow candidate lists of the substep's first density pass (L.cnt null: none);
// they are valid while no phase change re-sorted the sets.
__global__ void k_link_colour_warp(DevParams P, DevState* S, SetView vd, snowb_particle_data dem,
                                   const uint32_t* __restrict__ fs, const uint32_t* __restrict__ fe,
                                   const uint8_t* __restrict__ active, uint32_t colour, int dynamic, NList L,
                                   SCList sc)
{
    vd.n = S->n_dem;
    const bool lists = L.cnt != nullptr && S->changed == 0;
    const uint32_t qx = P.gsx >> 2, qy = P.gsy >> 2, qz = P.gsz >> 2;
    // the listed super-cells of this colour, or all of them
    const uint32_t total = sc.flag ? sc.count[colour] : qx * qy * qz;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < total; w += nwarps) {
        const uint32_t t = sc.flag ? sc.list[colour * sc.per + w] : w;
        const uint32_t sx = 2u * (t % qx) + (colour & 1u);
        const uint32_t sy = 2u * ((t / qx) % qy) + ((colour >> 1) & 1u);
        const uint32_t sz = 2u * (t / (qx * qy)) + ((colour >> 2) & 1u);
        // The 8 cells (dz, dy, dx) in hash order -- ascending sorted index -- with lane c
        // loading cell c's range; the super-cell's particles are then taken 32 at a time in
        // that order (cell by cell, ascending index), as the cell-by-cell loops would.
        uint32_t cb = 0, cn = 0;
        if (lane < 8u) {
            const uint32_t dz = lane >> 2, dy = (lane >> 1) & 1u, dx = lane & 1u;
            const uint32_t h = ((2u * sz + dz) * P.gsy + (2u * sy + dy)) * P.gsx + (2u * sx + dx);
            cb = fs[h];
            cn = fe[h] - cb;
        }
        uint32_t incl = cn;
#pragma unroll
        for (uint32_t o = 1; o < 8u; o <<= 1) {
            const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += v;
        }
        uint32_t st[8], bs[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            st[q] = __shfl_sync(0xffffffffu, incl - cn, q);   // first flattened position of cell q
            bs[q] = __shfl_sync(0xffffffffu, cb, q);
        }
        const uint32_t total_p = __shfl_sync(0xffffffffu, incl, 7);
        for (uint32_t f0 = 0; f0 < total_p; f0 += 32u) {
            const uint32_t f = f0 + lane;
            uint32_t i = 0;
            bool act = false;
            if (f < total_p) {
                // the last cell starting at or before f holds it (empty cells start where the
                // next one does)
                uint32_t s0 = st[0], b0 = bs[0];
#pragma unroll
                for (int r = 1; r < 8; ++r)
                    if (st[r] <= f) { s0 = st[r]; b0 = bs[r]; }
                i = b0 + (f - s0);
                act = active[i] != 0;
            }
            uint32_t am = __ballot_sync(0xffffffffu, act);
            while (am) {
                const int k = __ffs(am) - 1;
                am &= am - 1u;
                const uint32_t ii = __shfl_sync(0xffffffffu, i, k);
                const uint32_t lc = lists ? L.cnt[L.cap + ii] : NL_OVF;
                if (lc & NL_OVF) link_particle_warp(P, vd, dem, ii, dynamic, S);
                else link_particle_list(P, vd, dem, ii, dynamic, S, L, lc & 1023u);
            }
        }
        if (sc.flag && lane == 0) sc.flag[colour * sc.per + t] = 0u;   // ready for the next pass
    }
}
// general maximum_connection: the plain restatement with every access in memory
__device__ void link_particle(const DevParams& P, const SetView& vd, const snowb_particle_data& d, uint32_t i,
                              int dynamic, DevState* S)
{
    const uint32_t M = P.maxc;
    const float3 p = vd.pos(i);
    const uint32_t o = vd.gi[i];
    const GCell g = grid_pos(P, p, vd.scene(i));
    const float T = d.T[o];
    FOR27 {
        uint32_t s, e;
        if (!vd.range(P, g, ox, oy, oz, s, e)) continue;
        for (uint32_t j = s; j < e; ++j) {
            if (j == i) continue;
            const uint32_t o1 = vd.gi[j];
            const float dist = len3(sub3(p, vd.pos(j)));
            const uint32_t count = d.iter_end[o] - o * M;
            const uint32_t tol = link_tolerance(P, T, dynamic);
            if (dist < P.h && count < tol) {
                bool dup = false;
                for (uint32_t q = M * o; q < M * (o + 1); ++q)
                    if (d.connect_record[q] == o1) { dup = true; break; }
                if (dup) break;   // the reference returns from the cell helper
                for (uint32_t q = M * o; q < M * (o + 1); ++q) {
                    if (d.connect_record[q] == SNOWB_UMAX) {
                        d.connect_record[q] = o1;
                        bool valid = false;
                        if (d.iter_end[o1] < (o1 + 1) * M)
                            for (uint32_t r = o1 * M; r < (o1 + 1) * M; ++r)
                                if (d.connect_record[r] == SNOWB_UMAX) {
                                    d.connect_record[r] = o;
                                    d.connect_length[r] = dist;
                                    d.iter_end[o1]++;
                                    if (o1 >= vd.n) atomicOr(&S->tail_dirty, 1u);
                                    valid = true;
                                    break;
                                }
                        if (valid) { d.connect_length[q] = dist; d.iter_end[o]++; atomicAdd(&S->n_links, 1u); }
                        else d.connect_record[q] = SNOWB_UMAX;
                        break;
                    }
                }
            }
        }
    }
}
// Link formation's copy of the snow set's sorted view (the arrays its passes read: the
// sorted copies, grid index and hash, the cell table and the sort's cell offsets), taken
// after the sort point before it, so that the first iteration's sort point may rewrite the
// set's view while link formation runs.  `full` entries of the particle arrays (the
// caller's arrays hold that many), `ncells` of the cell table.
__global__ void k_copy_link_view(SetView v, uint32_t full, uint32_t ncells, const uint32_t* __restrict__ off,
                                 float4* __restrict__ p4, snowb_float3* __restrict__ sp, uint32_t* __restrict__ gi,
                                 uint32_t* __restrict__ gh, uint32_t* __restrict__ sid, uint32_t* __restrict__ cs,
                                 uint32_t* __restrict__ ce, uint32_t* __restrict__ off_o)
{
    const uint32_t m = full > ncells + 1 ? full : ncells + 1;
    GRID_LOOP(k, m) {
        if (k < full) {
            p4[k] = v.p4[k];
            sp[k] = v.sp[k];
            gi[k] = v.gi[k];
            gh[k] = v.gh[k];
            if (v.sid) sid[k] = v.sid[k];
        }
        if (k < ncells) { cs[k] = v.cs[k]; ce[k] = v.ce[k]; }
        if (k <= ncells) off_o[k] = off[k];
    }
}
// one colour: one thread per super-cell of that colour; fs/fe give each hash cell's
// current (non-stale) sorted range
__global__ void k_link_colour(DevParams P, DevState* S, SetView vd, snowb_particle_data dem,
                              const uint32_t* __restrict__ fs, const uint32_t* __restrict__ fe,
                              const uint8_t* __restrict__ active, uint32_t colour, int dynamic)
{
    vd.n = S->n_dem;
    const uint32_t qx = P.gsx >> 2, qy = P.gsy >> 2, qz = P.gsz >> 2;
    const uint32_t total = qx * qy * qz;
    GRID_LOOP(t, total) {
        const uint32_t sx = 2u * (t % qx) + (colour & 1u);
        const uint32_t sy = 2u * ((t / qx) % qy) + ((colour >> 1) & 1u);
        const uint32_t sz = 2u * (t / (qx * qy)) + ((colour >> 2) & 1u);
        for (uint32_t dz = 0; dz < 2; ++dz)
            for (uint32_t dy = 0; dy < 2; ++dy)
                for (uint32_t dx = 0; dx < 2; ++dx) {
                    const uint32_t h = ((2u * sz + dz) * P.gsy + (2u * sy + dy)) * P.gsx + (2u * sx + dx);
                    const uint32_t b = fs[h], e = fe[h];
                    for (uint32_t i = b; i < e; ++i)
                        if (active[i]) {
                            if (P.maxc <= SNOWB_MAXC_FAST) link_particle_fast(P, vd, dem, i, dynamic, S);
                            else link_particle(P, vd, dem, i, dynamic, S);
                        }
                }
    }
}
// adjust_connections_d (:4768-4808) in ascending index order (single thread).  The
// reference indexes the partner's slots with an empty record once the count exceeds the
// cap (an out-of-bounds read); that partner loop is skipped here.
__global__ void k_adjust_links(DevParams P, DevState* S, snowb_particle_data d, uint32_t full)
{
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    const uint32_t n = S->n_dem, M = P.maxc;
    for (uint32_t i = 0; i < n; ++i) {
        uint32_t cm = __float2uint_rz(((d.T[i] - P.Tf) / (P.Th - P.Tf)) * (float)M);
        if (cm > M) cm = M;
        uint32_t count = 0;
        for (uint32_t s = M * i; s < M * (i + 1); ++s) {
            count = d.connect_record[s] != SNOWB_UMAX ? count + 1 : count;
            if (count > cm) {
                const uint32_t j = d.connect_record[s];
                d.connect_record[s] = SNOWB_UMAX;
                d.connect_length[s] = 0.f;
                d.iter_end[i]--;
                if (j == SNOWB_UMAX || j >= full) continue;
                if (j >= n) S->tail_dirty = 1u;
                for (uint32_t q = M * j; q < M * (j + 1); ++q)
                    if (d.connect_record[q] == i) {
                        d.connect_record[q] = SNOWB_UMAX; d.connect_length[q] = 0.f; d.iter_end[j]--;
                    }
            }
        }
    }
}

}  // namespace snowb
