// Test helper: sequential host emulation of the CUDA Delaunay pipeline.
// Every data-parallel phase of the device code runs here as a loop over its
// items, calling the same __host__ __device__ functions
// (cuda-stereo-matching_b200/csrc/delaunay_core.h), so the algorithm can be
// checked on the CPU against the exact checker and Triangle.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <unordered_map>
#include <vector>

#include "../../cuda-stereo-matching_b200/csrc/delaunay_core.h"

using namespace elas::del;

// px, py: n points; row_off: nrows+1 offsets of points per lattice row
// (points of a row share y).  tris_out: capacity cap triangles.  Returns the
// triangle count, or -1 on an internal error.  stats (nullable):
// [0] rounds, [1] flips.
extern "C" int emu_delaunay(const int32_t* px, const int32_t* py, int n, const int32_t* row_off,
                            int nrows, int32_t* tris_out, int cap, long long* stats) {
    Pts P{px, py};
    // 1. per-row sort + dedup
    std::vector<std::vector<int32_t>> rows(nrows);
    for (int r = 0; r < nrows; ++r) {
        std::vector<int32_t> v;
        for (int i = row_off[r]; i < row_off[r + 1]; ++i) v.push_back(i);
        std::sort(v.begin(), v.end(), [&](int a, int b) {
            return px[a] != px[b] ? px[a] < px[b] : a < b;
        });
        for (size_t k = 0; k < v.size(); ++k)
            if (k == 0 || px[v[k]] != px[v[k - 1]]) rows[r].push_back(v[k]);
    }
    std::vector<int> ne;
    for (int r = 0; r < nrows; ++r)
        if (!rows[r].empty()) ne.push_back(r);
    int Tmax = 2 * n + 8;
    std::vector<int32_t> tri(3 * size_t(Tmax)), opp(3 * size_t(Tmax)), fwd(3 * size_t(Tmax), -1),
        cand(2 * size_t(Tmax));
    std::vector<uint32_t> lock(Tmax, LOCK_FREE);
    int32_t ctr[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    int T = 0;
    // 2. strips
    for (size_t s = 0; s + 1 < ne.size(); ++s) {
        auto& A = rows[ne[s]];
        auto& B = rows[ne[s + 1]];
        int cnt = int(A.size()) + int(B.size()) - 2;
        if (T + cnt > Tmax) return -1;
        zipper(P, A.data(), int(A.size()), B.data(), int(B.size()), &tri[3 * size_t(T)]);
        T += cnt;
    }
    // 3. pockets
    if (ne.size() >= 2) {
        std::vector<int32_t> chain(ne.size()), stack(ne.size());
        for (size_t s = 0; s < ne.size(); ++s) chain[s] = rows[ne[s]].front();
        T += fill_pockets(P, chain.data(), int(chain.size()), +1, stack.data(), &tri[3 * size_t(T)]);
        for (size_t s = 0; s < ne.size(); ++s) chain[s] = rows[ne[s]].back();
        T += fill_pockets(P, chain.data(), int(chain.size()), -1, stack.data(), &tri[3 * size_t(T)]);
    }
    if (T > Tmax) return -1;
    // 4. adjacency
    std::unordered_map<uint64_t, std::vector<int>> edges;
    for (int h = 0; h < 3 * T; ++h) {
        int t = h / 3, s = h % 3;
        edges[edge_key(tri[3 * t + s], tri[3 * t + (s + 1) % 3])].push_back(h);
    }
    for (auto& kv : edges) {
        if (kv.second.size() == 1) opp[kv.second[0]] = -1;
        else if (kv.second.size() == 2) { opp[kv.second[0]] = kv.second[1]; opp[kv.second[1]] = kv.second[0]; }
        else return -1;
    }
    // 5. flip rounds
    Tri S{P, tri.data(), opp.data(), lock.data(), fwd.data(), cand.data(), ctr, Tmax};
    auto amin = [](uint32_t* p, uint32_t v) { if (v < *p) *p = v; };
    auto aadd = [](int32_t* p, int v) { int o = *p; *p += v; return o; };
    long long rounds = 0, flips = 0;
    for (uint32_t round = 0; round < 100000; ++round) {
        for (int t = 0; t < T; ++t)
            if (!flip_propose(S, t, T, round, amin, aadd)) return -1;
        int nc = ctr[2 + (round & 1)];
        ++rounds;
        if (nc == 0) break;
        for (int c = 0; c < nc; ++c) flips += flip_apply(S, cand[c], round) ? 1 : 0;
        for (int t = 0; t < T; ++t) flip_repair(S, t);
        ctr[2 + ((round + 1) & 1)] = 0;
    }
    for (int t = 0; t < T; ++t) normalise(&tri[3 * size_t(t)]);
    if (T <= cap) std::memcpy(tris_out, tri.data(), sizeof(int32_t) * 3 * size_t(T));
    if (stats) { stats[0] = rounds; stats[1] = flips; }
    return T;
}
