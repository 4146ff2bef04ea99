// Test helper: sequential host emulation of the CUDA Delaunay pipeline
// (cuda-stereo-matching_b200/csrc/k_delaunay.cu).  Every data-parallel
// phase of the device code runs here as a loop over its items and calls the
// same __host__ __device__ functions (delaunay_core.h), so the algorithm can
// be checked on the CPU against the exact checker and Triangle.
#include <algorithm>
#include <cstdlib>
#include <cstdint>
#include <cstring>
#include <unordered_map>
#include <vector>

#include "../../cuda-stereo-matching_b200/csrc/delaunay_core.h"

using namespace elas::del;

// px, py: n points; row_off: nrows+1 offsets of the points of each lattice
// row (points of a row share y).  tris_out: room for cap triangles.  Returns
// the triangle count, or -1 on an internal error.  stats (nullable):
// [0] flip rounds, [1] flips.
// phased = 0: rounds in the propose / flip / resolve / relink formulation
// with worklists (k_flip_global).  phased = 1: rounds in the three-phase
// formulation of k_flip_local and k_flip_smem (flip; resolve and propose
// the outer edges; relink and re-propose the lost proposals; two lock
// arrays by round parity).  Both must give the same triangles, in the same
// slots, after the same rounds and flips.
static int emu_core(const int32_t* px, const int32_t* py, int n, const int32_t* row_off, int nrows,
                    int32_t* tris_out, int cap, long long* stats, int phased) {
    Pts P{px, py};
    // 1. per-row sort + dedup (k_rowsort)
    std::vector<int32_t> srt(std::max(n, 1)), rcnt(nrows, 0);
    for (int r = 0; r < nrows; ++r) {
        std::vector<int32_t> v;
        for (int i = row_off[r]; i < row_off[r + 1]; ++i) v.push_back(i);
        std::sort(v.begin(), v.end(), [&](int a, int b) { return px[a] != px[b] ? px[a] < px[b] : a < b; });
        int m = 0;
        for (size_t k = 0; k < v.size(); ++k)
            if (k == 0 || px[v[k]] != px[v[k - 1]]) srt[row_off[r] + m++] = v[k];
        rcnt[r] = m;
    }
    // 2. plan (k_plan)
    std::vector<int> ne, soff;
    for (int r = 0; r < nrows; ++r)
        if (rcnt[r] > 0) ne.push_back(r);
    const int R = int(ne.size());
    int off = 0;
    for (int s = 0; s + 1 < R; ++s) { soff.push_back(off); off += rcnt[ne[s]] + rcnt[ne[s + 1]] - 2; }
    const int Tmax = 2 * n + 16;
    std::vector<int32_t> tri(3 * size_t(Tmax), -1);
    int T = 0;
    if (R >= 2) {
        if (off + 2 * R > Tmax) return -1;
        std::vector<int32_t> ci(R), cx(R), cy(R), stk(4 * size_t(R));
        int pockets = 0;
        for (int side = 0; side < 2; ++side) {
            for (int s = 0; s < R; ++s) {
                int r = ne[s];
                int i = srt[row_off[r] + (side ? rcnt[r] - 1 : 0)];
                ci[s] = i; cx[s] = px[i]; cy[s] = py[i];
            }
            pockets += fill_pockets(ci.data(), cx.data(), cy.data(), R, side ? -1 : +1, stk.data(),
                                    &tri[3 * size_t(off + pockets)]);
        }
        T = off + pockets;
        // 3. strips (k_strips), every point of every non-empty row
        for (int lo = 0; lo < R; ++lo) {
            int r = ne[lo];
            const int32_t* A = &srt[row_off[r]];
            for (int k = 1; k < rcnt[r]; ++k) {
                int32_t t3[3];
                if (lo + 1 < R) {
                    int rb = ne[lo + 1];
                    int pos = strip_tri_upper(P, A, &srt[row_off[rb]], rcnt[rb], k, t3);
                    std::memcpy(&tri[3 * size_t(soff[lo] + pos)], t3, 12);
                }
                if (lo >= 1) {
                    int ra = ne[lo - 1];
                    int pos = strip_tri_lower(P, &srt[row_off[ra]], rcnt[ra], A, k, t3);
                    std::memcpy(&tri[3 * size_t(soff[lo - 1] + pos)], t3, 12);
                }
            }
        }
    }
    for (int i = 0; i < 3 * T; ++i)
        if (tri[i] < 0) return -1;   // a strip slot nobody wrote
    // 4. adjacency (k_hash_insert + k_link)
    std::vector<int32_t> opp(3 * size_t(Tmax), -1);
    std::unordered_map<uint64_t, std::vector<int>> edges;
    for (int h = 0; h < 3 * T; ++h) {
        int t = h / 3, s = h % 3;
        edges[edge_key(tri[3 * t + s], tri[3 * t + (s + 1) % 3])].push_back(h);
    }
    for (auto& kv : edges) {
        if (kv.second.size() == 2) { opp[kv.second[0]] = kv.second[1]; opp[kv.second[1]] = kv.second[0]; }
        else if (kv.second.size() != 1) return -1;
    }
    // 5. flips (k_flip_local / k_flip_smem / k_flip_global)
    std::vector<uint32_t> txy(3 * size_t(Tmax)), lock(Tmax, LOCK_FREE);
    std::vector<int32_t> fround(Tmax, -1), cand(6 * size_t(Tmax)), flips(6 * size_t(Tmax)), wl[2];
    wl[0].resize(6 * size_t(Tmax));
    wl[1].resize(6 * size_t(Tmax));
    for (int i = 0; i < 3 * T; ++i) txy[i] = pack_xy(px[tri[i]], py[tri[i]]);
    auto amin = [](uint32_t* p, uint32_t v) { if (v < *p) *p = v; };
    FlatTri<decltype(amin)> m{tri.data(), txy.data(), opp.data(), lock.data(), fround.data(), amin};
    std::vector<char> mark(3 * size_t(T), 0);
    int n_cur = 3 * T;
    long long rounds = 0, nflips = 0;
    if (phased) {
        std::vector<uint32_t> lock1(Tmax, LOCK_FREE);
        std::vector<int32_t> cl[2];
        // round 0's proposals: every interior edge once (owner rule), with lock array 0
        m.tlock = lock.data();
        for (int h = 0; h < 3 * T; ++h)
            if (!flip_propose(m, h, T, 0u, true, [&](int hh, int nn) { cl[0].push_back(hh); cl[0].push_back(nn); }))
                return -1;
        for (int round = 0; round < 100000; ++round) {
            const int cur = round & 1, nxt = cur ^ 1;
            std::vector<int32_t>& cc = cl[cur];
            std::vector<int32_t>& cn = cl[nxt];
            uint32_t* lock_cur = cur ? lock1.data() : lock.data();
            uint32_t* lock_nxt = cur ? lock.data() : lock1.data();
            rounds = round + 1;
            if (cc.empty()) break;
            // B: flip the winners; release the previous round's locks (list cn); clear the bitset
            m.tlock = lock_cur;
            int nf = 0;
            for (size_t c = 0; c < cc.size(); c += 2)
                if (flip_apply(m, cc[c], cc[c + 1], uint32_t(round))) {
                    flips[6 * nf] = cc[c] / 3;
                    flips[6 * nf + 1] = cc[c + 1];
                    ++nf;
                }
            for (size_t c = 0; c < cn.size(); c += 2) {
                lock_nxt[cn[c] / 3] = LOCK_FREE;
                lock_nxt[cn[c + 1]] = LOCK_FREE;
            }
            cn.clear();
            std::fill(mark.begin(), mark.end(), 0);
            auto propose_next = [&](int h, int nn) {
                const uint32_t p = prio(uint32_t(h), uint32_t(round + 1));
                if (p < lock_nxt[h / 3]) lock_nxt[h / 3] = p;
                if (p < lock_nxt[nn]) lock_nxt[nn] = p;
                cn.push_back(h);
                cn.push_back(nn);
            };
            // C1: resolve every flipped pair's outer neighbours, then test and
            // propose the outer edges (vertices are final after B)
            for (int f = 0; f < nf; ++f)
                for (int k = 0; k < 4; ++k) {
                    int r = flip_resolve_slot(m, outer_slot(flips[6 * f], flips[6 * f + 1], k), uint32_t(round), T);
                    if (r == -2) return -1;
                    flips[6 * f + 2 + k] = r;
                }
            for (int f = 0; f < nf; ++f)
                for (int k = 0; k < 4; ++k) {
                    const int x = outer_slot(flips[6 * f], flips[6 * f + 1], k), r = flips[6 * f + 2 + k];
                    if (r < 0) continue;
                    const int c = std::min(x, r), tw = c == x ? r : x;
                    if (mark[c]) continue;
                    mark[c] = 1;
                    if (edge_flippable(m, c, tw)) propose_next(c, tw / 3);
                }
            // C2: relink; re-propose the lost proposals without a new test
            for (int f = 0; f < nf; ++f) flip_relink(m, flips[6 * f], flips[6 * f + 1], &flips[6 * f + 2]);
            for (size_t c = 0; c < cc.size(); c += 2) {
                const int h = cc[c], n2 = cc[c + 1], t = h / 3;
                if (fround[t] != round && fround[n2] != round) propose_next(h, n2);
            }
            nflips += nf;
        }
        n_cur = 0;
    }
    for (int round = 0; !phased && round < 100000; ++round) {
        const std::vector<int32_t>& cur = wl[round & 1];
        std::vector<int32_t>& nxt = wl[(round + 1) & 1];
        int nc = 0;
        for (int k = 0; k < n_cur; ++k) {
            int h = round == 0 ? k : cur[k];
            if (!flip_propose(m, h, T, uint32_t(round), round == 0, [&](int hh, int nn) {
                    cand[2 * nc] = hh; cand[2 * nc + 1] = nn; ++nc;
                }))
                return -1;
        }
        ++rounds;
        if (nc == 0) break;
        int nf = 0;
        for (int c = 0; c < nc; ++c)
            if (flip_apply(m, cand[2 * c], cand[2 * c + 1], uint32_t(round))) {
                flips[6 * nf] = cand[2 * c] / 3;
                flips[6 * nf + 1] = cand[2 * c + 1];
                ++nf;
            }
        for (int f = 0; f < nf; ++f)
            for (int k = 0; k < 4; ++k) {
                int r = flip_resolve_slot(m, outer_slot(flips[6 * f], flips[6 * f + 1], k), uint32_t(round), T);
                if (r == -2) return -1;
                flips[6 * f + 2 + k] = r;
            }
        // the next worklist holds each interior edge once, as its lower half-edge
        int nn = 0;
        std::fill(mark.begin(), mark.end(), 0);
        auto push = [&](int x, int r) {
            if (r < 0) return;
            const int c = std::min(x, r);
            if (mark[c]) return;
            mark[c] = 1;
            nxt[nn++] = c;
        };
        for (int f = 0; f < nf; ++f) {
            int t = flips[6 * f], n2 = flips[6 * f + 1];
            flip_relink(m, t, n2, &flips[6 * f + 2]);
            for (int k = 0; k < 4; ++k) push(outer_slot(t, n2, k), flips[6 * f + 2 + k]);
        }
        for (int c = 0; c < nc; ++c) {
            int h = cand[2 * c], n2 = cand[2 * c + 1], t = h / 3;
            lock[t] = LOCK_FREE;
            lock[n2] = LOCK_FREE;
            if (fround[t] != round && fround[n2] != round) push(h, opp[h]);
        }
        nflips += nf;
        n_cur = nn;
    }
    for (int t = 0; t < T; ++t) normalise(&tri[3 * size_t(t)]);
    if (T <= cap) std::memcpy(tris_out, tri.data(), sizeof(int32_t) * 3 * size_t(T));
    if (stats) { stats[0] = rounds; stats[1] = nflips; }
    return T;
}

extern "C" int emu_delaunay(const int32_t* px, const int32_t* py, int n, const int32_t* row_off, int nrows,
                            int32_t* tris_out, int cap, long long* stats) {
    return emu_core(px, py, n, row_off, nrows, tris_out, cap, stats, 0);
}

extern "C" int emu_delaunay_phased(const int32_t* px, const int32_t* py, int n, const int32_t* row_off, int nrows,
                                   int32_t* tris_out, int cap, long long* stats) {
    return emu_core(px, py, n, row_off, nrows, tris_out, cap, stats, 1);
}

// Star construction (k_hull, k_star, k_star_scan, k_star_emit),
// sequentially: the same rows, hull boundary, windows, walk and owner rule,
// one point after another, each search a plain loop under the star order.  Triangles come out in point
// order, as on the device.  stats (nullable): [0] phase-2 searches, [1]
// squares grown, [2] candidates examined outside the staged windows.
// Returns the triangle count, or -1.
extern "C" int emu_delaunay_star(const int32_t* px, const int32_t* py, int n, const int32_t* row_off, int nrows,
                                 int32_t* tris_out, int cap, long long* stats) {
    // rows sorted by (x, index), repeated x dropped (k_rowsort)
    std::vector<int32_t> srt(std::max(n, 1)), rcnt(nrows, 0);
    std::vector<uint32_t> pxy(std::max(n, 1), PXY_NONE), sxy(std::max(n, 1), 0);
    for (int r = 0; r < nrows; ++r) {
        std::vector<int32_t> v;
        for (int i = row_off[r]; i < row_off[r + 1]; ++i) v.push_back(i);
        std::sort(v.begin(), v.end(), [&](int a, int b) { return px[a] != px[b] ? px[a] < px[b] : a < b; });
        int m = 0;
        for (size_t k = 0; k < v.size(); ++k)
            if (k == 0 || px[v[k]] != px[v[k - 1]]) {
                srt[row_off[r] + m] = v[k];
                sxy[row_off[r] + m] = pxy[v[k]] = pack_xy(px[v[k]], py[v[k]]);
                ++m;
            }
        rcnt[r] = m;
    }
    std::vector<int> ne;
    for (int r = 0; r < nrows; ++r)
        if (rcnt[r] > 0) ne.push_back(r);
    // hull boundary and the box of all points (k_hull)
    std::vector<int32_t> hnext(std::max(n, 1), -1), hprev(std::max(n, 1), -1);
    int32_t box[4] = {0, 0, 0, 0};
    const int R = int(ne.size());
    if (R >= 1) {
        box[0] = px[srt[row_off[ne[0]]]];
        box[2] = px[srt[row_off[ne[0]] + rcnt[ne[0]] - 1]];
        for (int s2 = 0; s2 < R; ++s2) {
            box[0] = std::min(box[0], px[srt[row_off[ne[s2]]]]);
            box[2] = std::max(box[2], px[srt[row_off[ne[s2]] + rcnt[ne[s2]] - 1]]);
        }
        box[1] = py[row_off[ne[0]]];
        box[3] = py[row_off[ne[R - 1]]];
    }
    if (R >= 2) {
        std::vector<int32_t> lst(R), rst(R);
        int nl = 0, nr = 0;
        auto first = [&](int s2) { return srt[row_off[ne[s2]]]; };
        auto last = [&](int s2) { return srt[row_off[ne[s2]] + rcnt[ne[s2]] - 1]; };
        std::vector<uint32_t> xyf(R), xyl(R);
        for (int s2 = 0; s2 < R; ++s2) {
            xyf[s2] = pxy[first(s2)];
            xyl[s2] = pxy[last(s2)];
        }
        hull_chain(0, R, xyf.data(), lst.data(), &nl);
        hull_chain(1, R, xyl.data(), rst.data(), &nr);
        const int tl = rcnt[ne[0]], bl = rcnt[ne[R - 1]];
        const int C = hull_cycle_len(tl, bl, nl, nr);
        auto at = [&](int j) {
            int row, pos;
            bool lastp;
            hull_cycle_at(j, R, tl, bl, lst.data(), nl, rst.data(), nr, &row, &pos, &lastp);
            return lastp ? last(row) : srt[row_off[ne[row]] + pos];
        };
        for (int j = 0; j < C; ++j) {
            hnext[at(j)] = at(j + 1 == C ? 0 : j + 1);
            hprev[at(j)] = at(j == 0 ? C - 1 : j - 1);
        }
    }
    long long circles = 0, squares = 0, evals = 0;
    const int R0 = star_r0(box, n);
    std::vector<int32_t> tri, ccw(STAR_NB), cw(STAR_NB);
    std::vector<std::pair<int32_t, uint32_t>> win;
    // every point of a region, row by row (the device splits them over lanes)
    auto each_in = [&](const StarRegion& g, auto&& take) {
        for (int r : ne) {
            const int32_t y = py[row_off[r]];
            if (y < g.y0 || y > g.y1) continue;
            int32_t x0, x1, x2, x3;
            g.cols2(y, box, &x0, &x1, &x2, &x3);
            for (int j = row_off[r]; j < row_off[r] + rcnt[r]; ++j) {
                const int32_t x = px_of(sxy[j]);
                if ((x >= x0 && x <= x1) || (x >= x2 && x <= x3)) {
                    ++evals;
                    take(srt[j], sxy[j]);
                }
            }
        }
    };
    for (int p = 0; p < n; ++p) {
        const uint32_t pp = pxy[p];
        if (pp == PXY_NONE) continue;
        const int32_t x0 = px_of(pp), y0 = py_of(pp);
        auto covers = [&](int Rs) {
            return x0 - Rs <= box[0] && x0 + Rs >= box[2] && y0 - Rs <= box[1] && y0 + Rs >= box[3];
        };
        // the window: staged once, grown (persisting for the point's later
        // searches) while its rings fit STAR_CAP
        win.clear();
        each_in(star_square_region(pp, R0, box), [&](int32_t s2, uint32_t sx) { win.push_back({s2, sx}); });
        const bool staged = win.size() <= size_t(STAR_CAP);
        int Rw = R0;
        bool ring_full = !staged;
        // one window growth, its ring's points given to take; false once
        // the rings no longer fit (the ring was still searched)
        auto grow = [&](auto&& take) {
            ++squares;
            const size_t K0 = win.size();
            each_in(star_ring_region(pp, Rw, box), [&](int32_t s2, uint32_t sx) {
                take(s2, sx);
                win.push_back({s2, sx});
            });
            if (win.size() > size_t(STAR_CAP)) {
                win.resize(K0);
                ring_full = true;
                return false;
            }
            Rw *= 2;
            return true;
        };
        auto nearest = [&]() -> int {
            unsigned long long best = ~0ull;
            auto take = [&](int s2, uint32_t sx) {
                if (s2 == p) return;
                const int32_t dx = dx_p(sx, pp), dy = dy_p(sx, pp);
                best = std::min<unsigned long long>(best, uint64_t(uint32_t(dx * dx + dy * dy)) << 32 | uint32_t(s2));
            };
            for (auto& c : win) take(c.first, c.second);
            for (int Rs = Rw;;) {
                const uint64_t d2 = best >> 32;
                if (best != ~0ull && d2 <= uint64_t(Rs) * uint64_t(Rs)) return int(uint32_t(best));
                if (covers(Rs)) return best == ~0ull ? -1 : int(uint32_t(best));
                if (Rs == Rw && !ring_full) {
                    if (!grow(take)) Rs *= 2;
                    else Rs = Rw;
                    continue;
                }
                if (best != ~0ull) {
                    // the nearest lies within distance sqrt(d2): the square of that half-size
                    int d = int(std::sqrt(double(d2)));
                    while (uint64_t(d) * uint64_t(d) < d2) ++d;
                    ++circles;
                    best = ~0ull;
                    each_in(star_square_region(pp, d, box), take);
                    return int(uint32_t(best));
                }
                Rs = star_square(Rs);
                ++squares;
                each_in(star_square_region(pp, Rs, box), take);
            }
        };
        auto next = [&](int q, int side) -> int {
            const uint32_t pq = pxy[q];
            int bi = -1;
            uint32_t bxy = 0;
            auto take = [&](int s2, uint32_t sx) {
                if (!star_side(pp, pq, sx, side)) return;
                if (bi < 0 || star_better(p, pp, q, pq, bi, bxy, s2, sx, side)) {
                    bi = s2;
                    bxy = sx;
                }
            };
            for (auto& c : win) take(c.first, c.second);
            for (int Rs = Rw;;) {
                if (bi >= 0 && circle_inside(pp, pq, bxy, Rs, box)) return bi;
                if (covers(Rs)) return bi;
                if (Rs == Rw && !ring_full) {
                    if (!grow(take)) Rs *= 2;
                    else Rs = Rw;
                    continue;
                }
                int need = 0;
                if (bi >= 0) circle_within(pp, pq, bxy, Rs, box, &need);
                if (bi >= 0 && need <= 2 * Rs) {
                    ++circles;
                    each_in(star_circle_region(pp, pq, bxy, box), take);
                    return bi;
                }
                Rs = star_square(Rs);
                ++squares;
                each_in(star_half_region(pp, pq, side, Rs, box), take);
            }
        };
        int m = 0, k = 0;
        bool closed = false;
        if (!star_walk(hnext[p], hprev[p], nearest, next, ccw.data(), cw.data(), STAR_NB, &m, &k, &closed))
            return -1;
        const int deg = m + k, nt = star_tris(deg, closed);
        for (int i = 0; i < nt; ++i) {
            const int a = star_at(ccw.data(), m, cw.data(), k, i);
            const int b = star_at(ccw.data(), m, cw.data(), k, i + 1 == deg ? 0 : i + 1);
            if (p < a && p < b) {
                tri.push_back(p);
                tri.push_back(a);
                tri.push_back(b);
            }
        }
    }
    const int T = int(tri.size() / 3);
    if (T <= cap) std::memcpy(tris_out, tri.data(), sizeof(int32_t) * tri.size());
    if (stats) { stats[0] = circles; stats[1] = squares; stats[2] = evals; }
    return T;
}

// hull_chain (the stack walk) and hull_on_chain (the per-point test of the
// device) on one chain: returns 1 if they keep the same points.
extern "C" int emu_hull_agree(const int32_t* xs, const int32_t* ys, int R, int side) {
    std::vector<uint32_t> xy(std::max(R, 1));
    for (int i = 0; i < R; ++i) xy[i] = pack_xy(xs[i], ys[i]);
    std::vector<int32_t> st(std::max(R, 1));
    int n = 0;
    hull_chain(side, R, xy.data(), st.data(), &n);
    std::vector<char> keep(std::max(R, 1), 0);
    for (int j = 0; j < n; ++j) keep[st[j]] = 1;
    for (int i = 0; i < R; ++i)
        if (bool(keep[i]) != hull_on_chain(side, R, xy.data(), i)) return 0;
    return 1;
}

// The flip predicates on packed coordinates, for checks against exact
// integer arithmetic.  xy: (x, y) of a, b, c[, d].
extern "C" long long emu_orient_p(const int32_t* xy) {
    return orient_p(pack_xy(xy[0], xy[1]), pack_xy(xy[2], xy[3]), pack_xy(xy[4], xy[5]));
}
extern "C" long long emu_incircle_p(const int32_t* xy) {
    return incircle_p(pack_xy(xy[0], xy[1]), pack_xy(xy[2], xy[3]), pack_xy(xy[4], xy[5]), pack_xy(xy[6], xy[7]));
}
