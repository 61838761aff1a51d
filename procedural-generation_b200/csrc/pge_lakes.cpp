// The planet's lake balance on the host: ErosionState.refresh_lakes
// (globe/erosion/maps.py:422-479) with erosion.lake_fill off.
//
// The reference runs the hydro stage's own sequence on the eroding surface:
// the priority flood of the whole sphere with a FIFO for depression cells
// (globe/hydro/priority_flood.py:127-191, 294-318), D8 on the filled surface
// with flats draining to their flood parent (globe/hydro/routing.py:28-90,
// globe/hydro/d8.py:123-136), then the evaporation balance of every
// depression in one upstream-first accumulation (globe/hydro/balance.py:63-108,
// 159-284, depressions labelled by globe/hydro/lakes.py:18-46).  Every step
// after the flood follows the flood's pop order, which is a strictly serial
// quantity (each pop depends on every earlier one), so this runs as one host
// pass between iterations, as the reference's does, every erosion.flood_every
// iterations; the device hands it the float32 surface and the sea mask and
// takes back the lake flags and the closed lakes' levels.
//
// The arithmetic mirrors the reference's types: surfaces and the filled
// surface in float32, slopes from float32 height differences over a float64
// step length, the balance in float64, the water surface and the depth tests
// in float32.  Compiled without floating-point contraction.  The flood is
// serial; the per-cell passes (D8, the runoff, the flags) run on the host's
// cores with OpenMP, each cell's result independent of the split.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "../../include/pgerosion.h"

namespace pge {
namespace {

constexpr int D8_DI[8] = {1, 1, 0, -1, -1, -1, 0, 1};
constexpr int D8_DJ[8] = {0, 1, 1, 1, 0, -1, -1, -1};

// cell ids are interior flat indices (f * N + i) * N + j; `owner` maps an extended cell to the
// extended flat index of the interior cell that owns it
struct Sphere {
    int N, H, NE;
    const int32_t *owner;

    int64_t neighbor(int64_t c, int k) const
    {
        const int64_t NN = (int64_t)N * N;
        const int f = (int)(c / NN);
        const int64_t rem = c - f * NN;
        const int i = (int)(rem / N), j = (int)(rem - (int64_t)i * N);
        const int64_t o = owner[((int64_t)f * NE + i + H + D8_DI[k]) * NE + j + H + D8_DJ[k]];
        const int64_t NE2 = (int64_t)NE * NE;
        const int f2 = (int)(o / NE2);
        const int64_t r2 = o - f2 * NE2;
        const int ei = (int)(r2 / NE), ej = (int)(r2 - (int64_t)ei * NE);
        return ((int64_t)f2 * N + (ei - H)) * N + (ej - H);
    }
    // all eight neighbours; a cell off the face's edge ring has them on its own face
    void neighbors(int64_t c, int64_t *out) const
    {
        const int64_t NN = (int64_t)N * N;
        const int64_t rem = c % NN;
        const int i = (int)(rem / N), j = (int)(rem % N);
        if (i >= 1 && i <= N - 2 && j >= 1 && j <= N - 2) {
            for (int k = 0; k < 8; k++) out[k] = c + (int64_t)D8_DI[k] * N + D8_DJ[k];
        } else {
            for (int k = 0; k < 8; k++) out[k] = neighbor(c, k);
        }
    }
    int code_towards(int64_t c, int64_t target) const
    {
        int64_t nb[8];
        neighbors(c, nb);
        for (int k = 0; k < 8; k++)
            if (nb[k] == target) return k;
        return -1;
    }
};

// The flood's heap orders cells by (level, push order).  Levels are float32 surfaces and fewer than 2^32 cells
// are ever pushed, so the pair packs into one unsigned 64-bit key: the level's bits mapped to an order-preserving
// unsigned integer (negative zero taken as zero, so equal levels tie as the float compare has them) over the push
// count.  A 4-ary min-heap of (key, cell) pops exactly the sequence a (level, push order) heap does.
inline uint64_t level_key(float level, int64_t seq)
{
    if (level == 0.0f) level = 0.0f;
    uint32_t u;
    std::memcpy(&u, &level, 4);
    u = (u & 0x80000000u) ? ~u : (u | 0x80000000u);
    return ((uint64_t)u << 32) | (uint64_t)(uint32_t)seq;
}

class LevelHeap {
  public:
    bool empty() const { return k_.empty(); }
    void push(uint64_t key, int64_t cell)
    {
        k_.push_back(key);
        c_.push_back(cell);
        size_t i = k_.size() - 1;
        while (i > 0) {
            const size_t p = (i - 1) >> 2;
            if (k_[p] <= key) break;
            k_[i] = k_[p];
            c_[i] = c_[p];
            i = p;
        }
        k_[i] = key;
        c_[i] = cell;
    }
    int64_t pop()
    {
        const int64_t top = c_[0];
        const uint64_t key = k_.back();
        const int64_t cell = c_.back();
        k_.pop_back();
        c_.pop_back();
        const size_t n = k_.size();
        if (n > 0) {
            size_t i = 0;
            while (true) {
                const size_t first = 4 * i + 1;
                if (first >= n) break;
                size_t m = first;
                const size_t last = first + 4 < n ? first + 4 : n;
                for (size_t j = first + 1; j < last; j++)
                    if (k_[j] < k_[m]) m = j;
                if (k_[m] >= key) break;
                k_[i] = k_[m];
                c_[i] = c_[m];
                i = m;
            }
            k_[i] = key;
            c_[i] = cell;
        }
        return top;
    }
    void reserve(size_t n)
    {
        k_.reserve(n);
        c_.reserve(n);
    }
    void clear()
    {
        k_.clear();
        c_.clear();
    }

  private:
    std::vector<uint64_t> k_;
    std::vector<int64_t> c_;
};

// priority flood: the filled surface, each cell's flood parent and the pop sequence; drains are
// the ocean cells (or the lowest cell when there is no ocean)
void flood(const Sphere &S, const float *surface, std::vector<uint8_t> &drain, std::vector<float> &filled,
           std::vector<int64_t> &parent, std::vector<int64_t> &order, std::vector<int64_t> &pop_seq)
{
    const int64_t M = (int64_t)6 * S.N * S.N;
    bool any = false;
    for (int64_t c = 0; c < M && !any; c++) any = drain[c] != 0;
    if (!any) {
        int64_t lo = 0;
        for (int64_t c = 1; c < M; c++)
            if (surface[c] < surface[lo]) lo = c;
        drain[lo] = 1;
    }
    filled.assign(surface, surface + M);
    parent.assign(M, -1);
    order.assign(M, -1);
    pop_seq.clear();
    pop_seq.reserve(M);
    // per-thread scratch kept between calls (a refresh every few iterations reuses its pages)
    static thread_local std::vector<uint8_t> visited_s;
    static thread_local LevelHeap heap_s;
    static thread_local std::vector<int64_t> fifo_s;
    std::vector<uint8_t> &visited = visited_s;
    LevelHeap &heap = heap_s;
    std::vector<int64_t> &fifo = fifo_s;
    visited.assign(M, 0);
    heap.clear();
    fifo.clear();
    int64_t seq = 0;
    for (int64_t c = 0; c < M; c++) {
        if (!drain[c]) continue;
        visited[c] = 1;
        int64_t nb[8];
        S.neighbors(c, nb);
        bool push = false;
        for (int k = 0; k < 8 && !push; k++) push = !drain[nb[k]];
        if (push) heap.push(level_key(surface[c], seq++), c);
    }
    size_t head = 0;
    const int64_t NN = (int64_t)S.N * S.N;
    while (head < fifo.size() || !heap.empty()) {
        int64_t c;
        if (head < fifo.size()) {
            c = fifo[head++];
            if (head == fifo.size()) {
                fifo.clear();
                head = 0;
            }
        } else {
            c = heap.pop();
        }
        const float lvl = filled[c];
        order[c] = (int64_t)pop_seq.size();
        pop_seq.push_back(c);
        const int64_t f = c / NN;
        int64_t nb[8];
        S.neighbors(c, nb);
        for (int k = 0; k < 8; k++) {
            const int64_t n = nb[k];
            if (visited[n]) continue;
            // across a face edge the nearest-cell mapping can be one-sided: only reversible links
            if (n / NN != f && S.code_towards(n, c) < 0) continue;
            visited[n] = 1;
            parent[n] = c;
            if (surface[n] <= lvl) {
                filled[n] = lvl;
                fifo.push_back(n);
            } else {
                filled[n] = surface[n];
                heap.push(level_key(surface[n], seq++), n);
            }
        }
    }
}

// D8 on the filled surface: steepest physical descent among strictly lower neighbours, else the
// flood parent; returns false when a land cell has no direction (the flood never reached it)
bool flow_down(const Sphere &S, const float *metric, const std::vector<float> &filled, const uint8_t *ocean,
               const std::vector<int64_t> &parent, std::vector<int64_t> &down)
{
    const int64_t M = (int64_t)6 * S.N * S.N, NN = (int64_t)S.N * S.N;
    down.assign(M, -1);
    int64_t unreached = 0;
#pragma omp parallel for schedule(static) reduction(+ : unreached)
    for (int64_t c = 0; c < M; c++) {
        if (ocean[c]) continue;
        const int64_t rem = c % NN;
        const int i = (int)(rem / S.N), j = (int)(rem % S.N);
        const float *g = metric + 3 * ((int64_t)(i + S.H) * S.NE + (j + S.H));
        const float hc = filled[c];
        int64_t nb[8];
        S.neighbors(c, nb);
        int best = -1;
        double best_s = 0.0;
        for (int k = 0; k < 8; k++) {
            const int64_t n = nb[k];
            const float hn = filled[n];
            if (hn < hc) {
                const double di = D8_DI[k], dj = D8_DJ[k];
                const double d2 = (double)g[0] * di * di + 2.0 * (double)g[1] * di * dj + (double)g[2] * dj * dj;
                const float dh = hc - hn;
                const double s = (double)dh / std::sqrt(d2);
                if (s > best_s) {
                    best_s = s;
                    best = k;
                }
            }
        }
        if (best < 0 && parent[c] >= 0) best = S.code_towards(c, parent[c]);
        if (best < 0)
            unreached++;
        else
            down[c] = nb[best];
    }
    return unreached == 0;
}

// 8-connected components of `mask` joining only cells of identical level, numbered by their lowest
// cell id
int64_t label_components(const Sphere &S, const std::vector<uint8_t> &mask, const std::vector<float> &level,
                         std::vector<int64_t> &labels)
{
    const int64_t M = (int64_t)mask.size();
    labels.assign(M, -1);
    static thread_local std::vector<int64_t> stack_s;
    std::vector<int64_t> &stack = stack_s;
    stack.clear();
    int64_t n = 0;
    for (int64_t s = 0; s < M; s++) {
        if (!mask[s] || labels[s] >= 0) continue;
        labels[s] = n;
        stack.push_back(s);
        while (!stack.empty()) {
            const int64_t c = stack.back();
            stack.pop_back();
            int64_t nb[8];
            S.neighbors(c, nb);
            for (int k = 0; k < 8; k++) {
                const int64_t q = nb[k];
                if (mask[q] && labels[q] < 0 && level[q] == level[c]) {
                    labels[q] = n;
                    stack.push_back(q);
                }
            }
        }
        n++;
    }
    return n;
}

double budyko(double aridity)
{
    const double a = aridity > 1e-9 ? aridity : 1e-9;
    return std::sqrt(a * std::tanh(1.0 / a) * (1.0 - std::exp(-a)));
}

// the planet pass's full-size scratch, one per calling thread, kept between refreshes: every array is
// reassigned before it is read, and the OpenMP loops reach it through references taken on the calling thread
struct LakeScratch {
    std::vector<uint8_t> drain, dep;
    std::vector<float> filled, water;
    std::vector<int64_t> parent, order, pop_seq, down, topo, lab, cells, outlet_lake;
    std::vector<double> w, wr, af, et, pe, acc, run;
    std::vector<uint8_t> olake, takes;
    std::vector<float> surf_after;
};
LakeScratch &lake_scratch()
{
    static thread_local LakeScratch s;
    return s;
}

// numpy's clip(x, lo, hi) for float64: max then min, each a plain compare (so -0.0 clipped at 0.0 is 0.0)
inline double clip(double x, double lo, double hi)
{
    const double m = x > lo ? x : lo;
    return m < hi ? m : hi;
}

// settle_lake_loads (maps.py:490-628): the loads the lakes kept laid over their floors, the lakes numbered
// for the kernel.  olake: the overflowing lakes of this refresh (interior cell ids); water / surf their level
// and the ground under them (float32); parent / order / pop_seq the flood they came from.  Writes F.lay,
// F.pending (dense), F.lake_id, F.lake_room, the totals; takes[c] = 1 on the cells of numbered lakes.
// Returns 0, or -1 when more lakes take load than F.lake_room_cap holds.
int settle_lake_loads(const Sphere &S, const std::vector<uint8_t> &olake, const std::vector<float> &water, const float *surf,
                      const std::vector<int64_t> &parent, const std::vector<int64_t> &order, const std::vector<int64_t> &pop_seq,
                      PgeLakeFill &F, std::vector<uint8_t> &takes)
{
    const int64_t M = (int64_t)6 * S.N * S.N;
    double *load = F.lake_load;
    int32_t *lake_id = F.lake_id;
    std::memset(F.lay, 0, sizeof(double) * M);
    std::memset(F.pending, 0, sizeof(double) * M);
    takes.assign(M, 0);
    F.parked = F.laid = F.stray = F.room = 0.0;
    F.lakes = 0;
    for (int64_t c = 0; c < M; c++) F.parked += load[c];
    // the lakes: cells joined at one water level, numbered by their lowest cell id
    std::vector<int64_t> lab;
    const int64_t n = label_components(S, olake, water, lab);
    // a load belongs to the lake it was parked in: this refresh's lake over its cell, else the heir of its
    // old lake (the lake of this refresh covering most of it; ties to the higher number), else a stockpile
    std::vector<double> have(n > 0 ? n : 1, 0.0);
    bool any_held = false;
    for (int64_t c = 0; c < M && !any_held; c++) any_held = load[c] > 0.0;
    if (any_held) {
        int32_t was_max = -1;
        for (int64_t c = 0; c < M; c++) was_max = lake_id[c] > was_max ? lake_id[c] : was_max;
        const int64_t n_was = (int64_t)was_max + 1;
        std::vector<int64_t> heir(n_was > 0 ? n_was : 1, -1);
        if (n > 0) {
            std::vector<int64_t> keys;
            for (int64_t c = 0; c < M; c++)
                if (lake_id[c] >= 0 && lab[c] >= 0) keys.push_back((int64_t)lake_id[c] * n + lab[c]);
            std::sort(keys.begin(), keys.end());
            // per old lake the (count, new lake) largest in that order
            std::vector<int64_t> best_cnt(n_was > 0 ? n_was : 1, -1);
            for (size_t t = 0; t < keys.size();) {
                size_t u = t;
                while (u < keys.size() && keys[u] == keys[t]) u++;
                const int64_t cnt = (int64_t)(u - t), old = keys[t] / n, nl = keys[t] % n;
                if (cnt >= best_cnt[old]) {  // keys ascend, so an equal count goes to the higher new lake
                    best_cnt[old] = cnt;
                    heir[old] = nl;
                }
                t = u;
            }
        }
        for (int64_t c = 0; c < M; c++) {
            if (!(load[c] > 0.0)) continue;
            const int64_t to = lab[c] >= 0 ? lab[c] : (lake_id[c] >= 0 ? heir[lake_id[c]] : -1);
            if (to >= 0) {
                have[to] += load[c];
            } else {  // its lake has drained altogether: on downstream as a stockpile
                F.pending[c] += load[c];
                F.stray += load[c];
            }
        }
    }
    for (int64_t c = 0; c < M; c++) lake_id[c] = -1;
    std::vector<int64_t> cells;
    for (int64_t c = 0; c < M; c++)
        if (lab[c] >= 0) cells.push_back(c);
    const int64_t K = (int64_t)cells.size();
    if (K > 0) {
        // the plain each lake fills towards: its water at the outlet, `grade` higher per flood step inside it
        std::vector<double> plain(M);
        for (int64_t c = 0; c < M; c++) plain[c] = (double)water[c];
        for (const int64_t c : pop_seq) {
            if (lab[c] < 0) continue;
            const int64_t q = parent[c];
            if (q >= 0 && lab[q] == lab[c]) plain[c] = plain[q] + F.grade;
        }
        std::vector<double> room(K), far(K);
        for (int64_t t = 0; t < K; t++) {
            const int64_t c = cells[t];
            const double w = (double)water[c] + F.rise, g = plain[c];
            const double r = (g <= w ? g : w) - (double)surf[c];
            room[t] = r >= 0.0 ? r : 0.0;
        }
        // each lake's outlet: its first popped cell; distances from it as the crow flies
        std::vector<int64_t> first(n, INT64_MAX), outlet(n, 0);
        for (const int64_t c : cells) first[lab[c]] = order[c] < first[lab[c]] ? order[c] : first[lab[c]];
        for (const int64_t c : cells)
            if (order[c] == first[lab[c]]) outlet[lab[c]] = c;
        for (int64_t t = 0; t < K; t++) {
            const double *a = F.centres + 3 * cells[t], *b = F.centres + 3 * outlet[lab[cells[t]]];
            const double dx = a[0] - b[0], dy = a[1] - b[1], dz = a[2] - b[2];
            far[t] = std::sqrt((dx * dx + dy * dy) + dz * dz);
        }
        // farthest from the outlet first within each lake (ties in cell order)
        std::vector<int64_t> o(K);
        for (int64_t t = 0; t < K; t++) o[t] = t;
        std::stable_sort(o.begin(), o.end(), [&](int64_t x, int64_t y) {
            const int64_t lx = lab[cells[x]], ly = lab[cells[y]];
            if (lx != ly) return lx < ly;
            return -far[x] < -far[y];
        });
        std::vector<int64_t> sc(K), L(K);
        std::vector<double> sr(K);
        for (int64_t t = 0; t < K; t++) {
            sc[t] = cells[o[t]];
            sr[t] = room[o[t]];
            L[t] = lab[sc[t]];
        }
        std::vector<int64_t> ptr(n, K);
        for (int64_t t = K; t-- > 0;) ptr[L[t]] = t;
        std::vector<double> csum(K);
        double run = 0.0;
        for (int64_t t = 0; t < K; t++) {
            run += sr[t];
            csum[t] = run;
        }
        std::vector<double> left(n, 0.0), laid(n, 0.0);
        for (int64_t t = 0; t < K; t++) {
            const int64_t p = ptr[L[t]];
            const double before = (csum[t] - sr[t]) - (csum[p] - sr[p]);  // room in the lake's cells laid first
            const double lay = clip(have[L[t]] - before, 0.0, sr[t]);
            F.lay[sc[t]] = lay;
            F.laid += lay;
            left[L[t]] += sr[t] - lay;
            laid[L[t]] += lay;
        }
        for (int64_t l = 0; l < n; l++) {
            const double over = have[l] - laid[l];  // rounding only: the apply holds a lake to its room
            if (over > 1e-9) {
                F.pending[sc[ptr[l]]] += over;
                F.stray += over;
            }
        }
        // a lake with a frozen cell takes nothing; the others with room left are numbered in order
        std::vector<uint8_t> warm(n, 1);
        const float ice = (float)F.ice_evap;
        for (const int64_t c : cells)
            if (F.evap[c] <= ice) warm[lab[c]] = 0;
        std::vector<int64_t> id(n, -1);
        int64_t nid = 0;
        for (int64_t l = 0; l < n; l++)
            if (warm[l] && left[l] > 0.0) id[l] = nid++;
        if (nid > F.lake_room_cap) return -1;
        for (int64_t l = 0; l < n; l++)
            if (id[l] >= 0) {
                F.lake_room[id[l]] = left[l];
                F.room += left[l];
            }
        for (const int64_t c : cells)
            if (id[lab[c]] >= 0) {
                takes[c] = 1;
                lake_id[c] = (int32_t)id[lab[c]];
            }
        F.lakes = nid;
    }
    if (F.lakes == 0 && F.lake_room_cap > 0) F.lake_room[0] = 0.0;  // the reference's one-entry zero room
    std::memset(load, 0, sizeof(double) * M);
    return 0;
}

}  // namespace

// returns 0, or -1 when a land cell got no flow direction
int lake_balance_host(int N, int H, const int32_t *owner, const float *metric, const float *cell_area, double cell_size_m,
                      const float *surface, const uint8_t *ocean_in, const float *precip, const float *pet, double lake_evap,
                      double land_evap, double min_depth, uint8_t *lake_flag, float *water_out, float *closed_level,
                      PgeLakeFill *fill, PgeLakeInfo *info)
{
    Sphere S{N, H, N + 2 * H, owner};
    const int64_t M = (int64_t)6 * N * N;
    LakeScratch &X = lake_scratch();
    std::vector<uint8_t> &drain = X.drain, &dep = X.dep;
    std::vector<float> &filled = X.filled, &water = X.water;
    std::vector<int64_t> &parent = X.parent, &order = X.order, &pop_seq = X.pop_seq, &down = X.down, &topo = X.topo;
    drain.assign(ocean_in, ocean_in + M);
    flood(S, surface, drain, filled, parent, order, pop_seq);
    if (!flow_down(S, metric, filled, ocean_in, parent, down)) return -1;
    // upstream first: the pop sequence reversed, without the ocean
    topo.clear();
    for (size_t t = pop_seq.size(); t-- > 0;)
        if (!ocean_in[pop_seq[t]]) topo.push_back(pop_seq[t]);

    PgeLakeInfo inf{};
    water.assign(filled.begin(), filled.end());
    dep.assign(M, 0);
    int64_t ndep = 0;
#pragma omp parallel for schedule(static) reduction(+ : ndep)
    for (int64_t c = 0; c < M; c++) {
        dep[c] = filled[c] > surface[c] && !ocean_in[c];
        ndep += dep[c];
    }
    const bool any_dep = ndep > 0;
    if ((lake_evap > 0.0 || land_evap > 0.0) && any_dep) {
        std::vector<int64_t> &lab = X.lab, &cells = X.cells;
        const int64_t n = label_components(S, dep, filled, lab);
        // a depression's cells by depth (ties in cell order)
        cells.clear();
        for (int64_t c = 0; c < M; c++)
            if (lab[c] >= 0) cells.push_back(c);
        std::stable_sort(cells.begin(), cells.end(), [&](int64_t a, int64_t b) {
            if (lab[a] != lab[b]) return lab[a] < lab[b];
            return surface[a] < surface[b];
        });
        const int64_t K = (int64_t)cells.size();
        std::vector<int64_t> ptr(n + 1, K);
        for (int64_t t = K; t-- > 0;) ptr[lab[cells[t]]] = t;
        std::vector<double> &w = X.w, &wr = X.wr, &af = X.af;
        w.resize(M);
        wr.resize(M);
        af.resize(M);
        const double cs2 = cell_size_m * cell_size_m;
#pragma omp parallel for schedule(static)
        for (int64_t c = 0; c < M; c++) {
            w[c] = (double)precip[c];
            af[c] = (double)cell_area[c] / cs2;
        }
        std::vector<double> per(K);
        double k_lake = lake_evap;
        const bool runoff = land_evap > 0.0;
        if (runoff) {
            // the land evaporates too: a cell's rain runs off in the share Budyko's curve leaves, and
            // open water loses the potential evaporation less what the land under it would have
            std::vector<double> &et = X.et, &pe = X.pe;
            et.resize(M);
            pe.resize(M);
#pragma omp parallel for schedule(static)
            for (int64_t c = 0; c < M; c++) {
                const double rain = w[c] / af[c];
                pe[c] = land_evap * (double)pet[c];
                et[c] = rain * budyko(pe[c] / (rain > 1e-9 ? rain : 1e-9));
                wr[c] = (rain - et[c]) * af[c];
            }
            for (int64_t t = 0; t < K; t++) per[t] = (pe[cells[t]] - et[cells[t]]) * af[cells[t]];
            k_lake = 1.0;
        } else {
            wr.assign(w.begin(), w.end());
            for (int64_t t = 0; t < K; t++) per[t] = (double)pet[cells[t]] * af[cells[t]];
        }
        // cumulative loss of each depression with the water at each cell's level
        std::vector<double> csum(K), cum(K), z(K);
        double run_sum = 0.0;
        for (int64_t t = 0; t < K; t++) {
            run_sum += per[t];
            csum[t] = run_sum;
            z[t] = (double)surface[cells[t]];
        }
        for (int64_t L = 0; L < n; L++) {
            const double before = L > 0 ? csum[ptr[L] - 1] : 0.0;
            for (int64_t t = ptr[L]; t < ptr[L + 1]; t++) cum[t] = csum[t] - before;
        }
        // the outlet: the depression's first popped cell
        std::vector<int64_t> outlet(n, -1);
        std::vector<int64_t> &outlet_lake = X.outlet_lake;
        outlet_lake.assign(M, -1);
        for (int64_t t = 0; t < K; t++) {
            const int64_t c = cells[t], L = lab[c];
            if (outlet[L] < 0 || order[c] < order[outlet[L]]) outlet[L] = c;
        }
        std::vector<double> spill(n), level(n, 0.0), outflow(n, 0.0);
        for (int64_t L = 0; L < n; L++) {
            outlet_lake[outlet[L]] = L;
            spill[L] = (double)filled[outlet[L]];
        }
        // one accumulation, upstream first, solving each depression as it passes its outlet
        std::vector<double> &acc = X.acc, &run = X.run;
        acc.assign(w.begin(), w.end());
        run.assign(wr.begin(), wr.end());
        for (const int64_t c : topo) {
            const int64_t L = outlet_lake[c];
            if (L >= 0) {
                const double inflow = run[c];
                const int64_t lo = ptr[L], hi = ptr[L + 1];
                if (inflow <= 0.0) {
                    level[L] = z[lo];
                    outflow[L] = 0.0;
                } else {
                    const double need = inflow / k_lake;
                    const int64_t i = std::lower_bound(cum.begin() + lo, cum.begin() + hi, need) - (cum.begin() + lo);
                    if (i >= hi - lo) {
                        level[L] = spill[L];
                        outflow[L] = inflow - k_lake * cum[hi - 1];
                    } else {
                        level[L] = z[lo + i];
                        outflow[L] = 0.0;
                    }
                }
                if (runoff)
                    acc[c] = inflow > 0.0 ? acc[c] * (outflow[L] / inflow) : 0.0;
                else
                    acc[c] = outflow[L];
                run[c] = outflow[L];
            }
            const int64_t d = down[c];
            if (d >= 0) {
                acc[d] += acc[c];
                run[d] += run[c];
            }
        }
        // a cell above its depression's balance level dries out
        water.assign(surface, surface + M);
        for (int64_t t = 0; t < K; t++) {
            const int64_t c = cells[t];
            const float lv = (float)level[lab[c]];
            if (lv > water[c]) water[c] = lv;
        }
        for (int64_t c = 0; c < M; c++)
            if (ocean_in[c]) water[c] = filled[c];
        inf.depressions = n;
        for (int64_t L = 0; L < n; L++) {
            const bool closed = outflow[L] <= 0.0;
            const bool wet = level[L] > z[ptr[L]];
            inf.overflowing += !closed;
            inf.closed += closed && wet;
            inf.dry += closed && !wet;
        }
    }
    // overflowing lakes are flagged; a lake drawn below its rim is a closed sea at its level
    const float depth = (float)min_depth, rim = 1e-4f;
    std::vector<uint8_t> &takes = X.takes;
    std::vector<float> &surf_after = X.surf_after;
    if (fill) {
        // erosion.lake_fill: the overflowing lakes take the loads parked on them, then only what stays deeper
        // than min_depth over the laid sediment is still a lake (maps.py:466-470)
        std::vector<uint8_t> &olake = X.olake;
        olake.assign(M, 0);
        for (int64_t c = 0; c < M; c++) {
            const bool lake = (float)(water[c] - surface[c]) > depth && !ocean_in[c];
            olake[c] = lake && !(water[c] < (float)(filled[c] - rim));
        }
        if (settle_lake_loads(S, olake, water, surface, parent, order, pop_seq, *fill, takes) != 0) return -2;
        surf_after.assign(surface, surface + M);
        for (int64_t c = 0; c < M; c++)
            if (fill->lay[c] != 0.0) surf_after[c] = (float)(fill->height[c] + (fill->sediment[c] + fill->lay[c]));
    }
    const float *surf2 = fill ? surf_after.data() : surface;
    int64_t nlake = 0, nclosed = 0;
#pragma omp parallel for schedule(static) reduction(+ : nlake, nclosed)
    for (int64_t c = 0; c < M; c++) {
        bool lake = (float)(water[c] - surface[c]) > depth && !ocean_in[c];
        const bool closed = lake && water[c] < (float)(filled[c] - rim);
        if (fill) lake = lake && (float)(water[c] - surf2[c]) > depth;
        lake_flag[c] = lake && !closed ? (fill && takes[c] ? 2 : 1) : 0;
        if (closed_level) closed_level[c] = closed && lake ? water[c] : NAN;
        nlake += lake;
        nclosed += closed && lake;
    }
    inf.lake_cells = nlake;
    inf.lake_cells_closed = nclosed;
    if (water_out) std::memcpy(water_out, water.data(), sizeof(float) * M);
    if (info) *info = inf;
    return 0;
}

// the sediment fill_basins lays into the closed basins of a fresh state (maps.py:1278-1326): the flood's
// surface graded `step` (cell units per cell) up from each basin's outlet along the flood tree, where the
// flood found a basin deeper than min_depth off the ocean
void basin_fill_host(int N, int H, const int32_t *owner, const float *surface, const uint8_t *ocean_in, double step, double min_depth,
                     double *add, uint8_t *basin_out, int64_t *basin_cells)
{
    Sphere S{N, H, N + 2 * H, owner};
    const int64_t M = (int64_t)6 * N * N;
    std::vector<uint8_t> drain(ocean_in, ocean_in + M);
    std::vector<float> filled;
    std::vector<int64_t> parent, order, pop_seq;
    flood(S, surface, drain, filled, parent, order, pop_seq);
    // every cell at least `step` above the cell that flooded it, parents before children (pop order)
    std::vector<double> g(surface, surface + M);
    for (const int64_t c : pop_seq) {
        const int64_t q = parent[c];
        if (q >= 0) {
            const double v = g[q] + step;
            if (v > g[c]) g[c] = v;
        }
    }
    const float depth = (float)min_depth;
    int64_t nb = 0;
#pragma omp parallel for schedule(static) reduction(+ : nb)
    for (int64_t c = 0; c < M; c++) {
        const bool basin = (float)(filled[c] - surface[c]) > depth && !ocean_in[c];
        const double a = g[c] - (double)surface[c];
        add[c] = basin ? (a > 0.0 ? a : 0.0) : 0.0;
        if (basin_out) basin_out[c] = basin ? 1 : 0;
        nb += basin;
    }
    if (basin_cells) *basin_cells = nb;
}

// the lakes of a window balanced against evaporation (maps.py:675-736, erosion.window_lake_evap > 0) on a
// W x W array: the flat flood (globe/hydro/priority_flood.py:193-270) from the inactive cells and the
// array's border, the window's rain accumulated down the flood tree (globe/zoom/bake.py:323-330), each
// depression (8-connected cells the flood fills more than 1e-6 above the surface, active) settled where
// its inflow meets lake_evap x evap summed over the water at each level; returns the flags (deeper than
// min_depth, active) and lowers the routing surface to the water on them
void window_lake_balance_host(int W, const float *surface, const uint8_t *active, const float *precip, const float *evap,
                              double lake_evap, double min_depth, double *route, uint8_t *lake, int64_t *counts)
{
    const int64_t M = (int64_t)W * W;
    std::vector<uint8_t> drain(M);
    for (int64_t c = 0; c < M; c++) {
        const int i = (int)(c / W), j = (int)(c % W);
        drain[c] = !active[c] || i == 0 || i == W - 1 || j == 0 || j == W - 1;
    }
    // the flat flood: the same FIFO + (level, push order) heap, neighbours inside the array
    std::vector<float> filled(surface, surface + M);
    std::vector<int64_t> parent(M, -1), pop_seq;
    pop_seq.reserve(M);
    std::vector<uint8_t> visited(M, 0);
    LevelHeap heap;
    std::vector<int64_t> fifo;
    int64_t seq = 0;
    auto nbr = [&](int64_t c, int k, int64_t &n) {
        const int i2 = (int)(c / W) + D8_DI[k], j2 = (int)(c % W) + D8_DJ[k];
        if (i2 < 0 || i2 >= W || j2 < 0 || j2 >= W) return false;
        n = (int64_t)i2 * W + j2;
        return true;
    };
    for (int64_t c = 0; c < M; c++) {
        if (!drain[c]) continue;
        visited[c] = 1;
        bool push = false;
        for (int k = 0; k < 8 && !push; k++) {
            int64_t n;
            if (nbr(c, k, n)) push = !drain[n];
        }
        if (push) heap.push(level_key(surface[c], seq++), c);
    }
    size_t head = 0;
    while (head < fifo.size() || !heap.empty()) {
        int64_t c;
        if (head < fifo.size()) {
            c = fifo[head++];
            if (head == fifo.size()) {
                fifo.clear();
                head = 0;
            }
        } else {
            c = heap.pop();
        }
        const float lvl = filled[c];
        pop_seq.push_back(c);
        for (int k = 0; k < 8; k++) {
            int64_t n;
            if (!nbr(c, k, n) || visited[n]) continue;
            visited[n] = 1;
            parent[n] = c;
            if (surface[n] <= lvl) {
                filled[n] = lvl;
                fifo.push_back(n);
            } else {
                filled[n] = surface[n];
                heap.push(level_key(surface[n], seq++), n);
            }
        }
    }
    // the rain accumulated down the flood tree, children before parents
    std::vector<double> acc(M);
    for (int64_t c = 0; c < M; c++) acc[c] = (double)precip[c];
    for (size_t k = pop_seq.size(); k-- > 0;) {
        const int64_t c = pop_seq[k], q = parent[c];
        if (q >= 0) acc[q] += acc[c];
    }
    // depressions: 8-connected, labelled 1.. in raster order of their first cell
    std::vector<int64_t> lab(M, 0), stack;
    int64_t n = 0;
    for (int64_t c = 0; c < M; c++) {
        const bool dep = filled[c] > (float)(surface[c] + 1e-6f) && active[c];
        lab[c] = dep ? -1 : 0;
    }
    for (int64_t s0 = 0; s0 < M; s0++) {
        if (lab[s0] != -1) continue;
        lab[s0] = ++n;
        stack.push_back(s0);
        while (!stack.empty()) {
            const int64_t c = stack.back();
            stack.pop_back();
            for (int k = 0; k < 8; k++) {
                int64_t q;
                if (nbr(c, k, q) && lab[q] == -1) {
                    lab[q] = n;
                    stack.push_back(q);
                }
            }
        }
    }
    int64_t nover = 0, nclosed = 0, ndry = 0;
    std::vector<double> water(M);
    for (int64_t c = 0; c < M; c++) water[c] = (double)surface[c];
    if (n > 0) {
        std::vector<int64_t> cells;
        for (int64_t c = 0; c < M; c++)
            if (lab[c] > 0) cells.push_back(c);
        std::stable_sort(cells.begin(), cells.end(), [&](int64_t a, int64_t b) {
            if (lab[a] != lab[b]) return lab[a] < lab[b];
            return surface[a] < surface[b];
        });
        const int64_t K = (int64_t)cells.size();
        std::vector<int64_t> ptr(n + 2, K);
        for (int64_t t = K; t-- > 0;) ptr[lab[cells[t]]] = t;
        ptr[0] = 0;
        // the evaporative demand with the water at each cell's level, cumulated over every depression in turn
        std::vector<double> demand(K), z(K);
        double run_sum = 0.0;
        for (int64_t t = 0; t < K; t++) {
            const double e = (double)evap[cells[t]];
            run_sum += lake_evap * (e > 0.0 ? e : 0.0);
            demand[t] = run_sum;
            z[t] = (double)surface[cells[t]];
        }
        std::vector<double> spill(n + 1, -INFINITY), inflow(n + 1, -INFINITY), level(n + 1, 0.0);
        for (int64_t t = 0; t < K; t++) {
            const int64_t c = cells[t], L = lab[c];
            if ((double)filled[c] > spill[L]) spill[L] = (double)filled[c];
            if (acc[c] > inflow[L]) inflow[L] = acc[c];
        }
        for (int64_t L = 1; L <= n; L++) {
            const int64_t a = ptr[L], b = ptr[L + 1];
            if (b <= a) continue;
            const double need = inflow[L], before = a > 0 ? demand[a - 1] : 0.0;
            if (need <= 0.0) {
                level[L] = z[a] - 1.0;
                ndry++;
            } else if (demand[b - 1] - before <= need) {
                level[L] = spill[L];  // cannot evaporate what arrives: still spills
                nover++;
            } else {
                int64_t i = 0;
                while (i < b - a && demand[a + i] - before < need) i++;  // the first level whose loss reaches the inflow
                level[L] = z[a + (i < b - a - 1 ? i : b - a - 1)];
                nclosed++;
            }
        }
        for (int64_t c = 0; c < M; c++)
            if (lab[c] > 0) water[c] = level[lab[c]];
    }
    int64_t nlake = 0;
    for (int64_t c = 0; c < M; c++) {
        const bool l = water[c] - (double)surface[c] > min_depth && active[c];
        lake[c] = l ? 1 : 0;
        nlake += l;
        if (l && water[c] < route[c]) route[c] = water[c];
    }
    if (counts) {
        counts[0] = n;
        counts[1] = nover;
        counts[2] = nclosed;
        counts[3] = ndry;
        counts[4] = nlake;
    }
}

}  // namespace pge
