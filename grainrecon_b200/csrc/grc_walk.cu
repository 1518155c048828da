// grc_walk.cu -- best-first region growth of grow_indexed_region.m, on the host.
//
// The walk is sequential: from the current voxel every unvisited in-mask neighbour of the
// 18-neighbourhood is scored and kept when it beats the map, and the walk moves to the kept
// voxel of highest completeness while that stays above seed_comp * (1 - drop_off).  Scores
// come from a caller-supplied function; the library's own (grc_grow_best_first) fills a
// per-voxel cache a block of voxels at a time on the GPU, since a voxel's score for one U does
// not depend on the region grown so far.
#include <cmath>
#include <cstdint>
#include <utility>
#include <vector>

#include "grainrecon_b200.h"

namespace {

// grow_indexed_region.m:50-52, in this order (it decides which kept voxel comes first on ties)
const int kNeigb[18][3] = {{1, 1, 0},  {1, -1, 0},  {1, 0, 1},   {1, 0, -1},  {1, 0, 0},  {0, 1, 0},
                           {0, -1, 0}, {0, 1, 1},   {0, 0, 1},   {0, -1, 1},  {0, 1, -1}, {0, 0, -1},
                           {0, -1, -1}, {-1, 1, 0}, {-1, -1, 0}, {-1, 0, 1}, {-1, 0, -1}, {-1, 0, 0}};

struct Kept {  // one row of neg_list: [xn yn zn C dis_median Nr_intersect]
    int32_t x, y, z;
    double c, d, n;
};

// MATLAB round: halves away from zero
double mround(double v) { return v < 0 ? -std::floor(-v + 0.5) : std::floor(v + 0.5); }

// The reference takes [pixdist, index] = max(neg_list(:,4)/seed_comp) over the kept list every
// step (:93-94): the first maximum in list order, NaN ignored.  A linear scan makes the walk
// O(steps x frontier); this tree over list positions keeps, per node, the largest key and its
// leftmost position, so the same answer costs O(log n) per list change.
class FirstMax {
  public:
    void set(size_t pos, double key) {  // key of list position pos (NaN counts as absent)
        if (pos >= cap_) grow(pos + 1);
        size_t i = pos + cap_;
        key_[i] = std::isnan(key) ? -INFINITY : key;
        nan_[i] = std::isnan(key);
        for (i >>= 1; i >= 1; i >>= 1) pull(i);
    }
    void clear(size_t pos) {  // position pos leaves the list
        size_t i = pos + cap_;
        key_[i] = -INFINITY;
        nan_[i] = false;
        for (i >>= 1; i >= 1; i >>= 1) pull(i);
    }
    // (key, position) of the first maximum among positions [0, n); key NaN when all are NaN
    std::pair<double, size_t> first_max(size_t n) const {
        if (key_[1] == -INFINITY) {  // nothing but NaN or -inf keys: the reference's max rules
            for (size_t p = 0; p < n; ++p)
                if (!nan_[p + cap_]) return {-INFINITY, p};
            return {NAN, 0};
        }
        return {key_[1], pos_[1]};
    }

  private:
    void pull(size_t i) {
        const size_t l = 2 * i, r = 2 * i + 1;
        const bool left = key_[l] >= key_[r];  // ties go to the leftmost position
        key_[i] = left ? key_[l] : key_[r];
        pos_[i] = left ? pos_[l] : pos_[r];
    }
    void grow(size_t need) {
        size_t cap = cap_ ? cap_ : 64;
        while (cap < need) cap *= 2;
        std::vector<double> key(2 * cap, -INFINITY);
        std::vector<size_t> pos(2 * cap, 0);
        std::vector<uint8_t> nan(2 * cap, 0);
        for (size_t p = 0; p < cap_; ++p) {
            key[cap + p] = key_[cap_ + p];
            nan[cap + p] = nan_[cap_ + p];
        }
        for (size_t p = 0; p < cap; ++p) pos[cap + p] = p;
        key_.swap(key);
        pos_.swap(pos);
        nan_.swap(nan);
        cap_ = cap;
        for (size_t i = cap_ - 1; i >= 1; --i) pull(i);
    }
    size_t cap_ = 0;
    std::vector<double> key_;
    std::vector<size_t> pos_;
    std::vector<uint8_t> nan_;
};

}  // namespace

extern "C" int grc_walk_best_first(grc_walk_score_fn score, void *user, int64_t X, int64_t Y, int64_t Z,
                                   const double *I, const double *Imask, const double *DisMedian,
                                   const double *Ninter, const int32_t seed[3], double drop_off, double maxD,
                                   double indexed_comp, double maxDmedian, double *C_out, double *D_out,
                                   double *N_out, uint8_t *J_out, int64_t *idx_out, int64_t idx_cap, int64_t *n_idx,
                                   double center[3], int *replace_center) {
    if (!score || !I || !Imask || !DisMedian || !Ninter || !seed || !C_out || !D_out || !N_out || !J_out ||
        !n_idx || !center || !replace_center || (idx_cap > 0 && !idx_out))
        return GRC_EINVAL;
    if (X < 1 || Y < 1 || Z < 1 || X > INT32_MAX || Y > INT32_MAX || Z > INT32_MAX) return GRC_EINVAL;
    int32_t x = seed[0], y = seed[1], z = seed[2];
    if (x < 1 || y < 1 || z < 1 || x > X || y > Y || z > Z) return GRC_EINVAL;
    const int64_t nvox = X * Y * Z;
    auto lin = [&](int64_t a, int64_t b, int64_t c) { return (a - 1) + X * ((b - 1) + Y * (c - 1)); };

    // grow_indexed_region.m:32-41: the seed takes indexed_comp; outputs start as the input maps
    std::vector<double> Iw(I, I + nvox);
    Iw[lin(x, y, z)] = indexed_comp;
    for (int64_t i = 0; i < nvox; ++i) {
        C_out[i] = Iw[i];
        D_out[i] = DisMedian[i];
        N_out[i] = Ninter[i];
        J_out[i] = 0;
    }
    const double seed_comp = Iw[lin(x, y, z)];
    double csum = seed_comp;
    double cpos[3] = {seed_comp * x, seed_comp * y, seed_comp * z};
    const double center0[3] = {cpos[0] / csum, cpos[1] / csum, cpos[2] / csum};
    int64_t n_mask = 0;
    for (int64_t i = 0; i < nvox; ++i) n_mask += Imask[i] > 0;

    std::vector<Kept> neg;
    FirstMax order;  // keys C / seed_comp of the kept list
    int32_t nb[18 * 3];
    double sc[18 * 3];
    int64_t reg_size = 0;
    for (;;) {
        // :61-86 -- unvisited in-mask neighbours, scored together, kept when they beat the map
        int n = 0;
        for (const auto &o : kNeigb) {
            const int64_t xn = x + o[0], yn = y + o[1], zn = z + o[2];
            if (xn < 1 || yn < 1 || zn < 1 || xn > X || yn > Y || zn > Z) continue;
            const int64_t k = lin(xn, yn, zn);
            if (J_out[k] != 0 || !(Imask[k] > 0)) continue;
            nb[3 * n] = (int32_t)xn;
            nb[3 * n + 1] = (int32_t)yn;
            nb[3 * n + 2] = (int32_t)zn;
            ++n;
        }
        if (n > 0) {
            const int rc = score(user, nb, n, sc);
            if (rc != GRC_OK) return rc;
            for (int j = 0; j < n; ++j) {
                const int64_t k = lin(nb[3 * j], nb[3 * j + 1], nb[3 * j + 2]);
                const double c = sc[3 * j + 1] / sc[3 * j];  // Nr_intersect / Nr_simu
                const double dmin = std::fmin(DisMedian[k], maxDmedian);  // MATLAB min ignores NaN
                if ((c > Iw[k] && sc[3 * j + 2] <= dmin) || (std::fabs(c - Iw[k]) <= 0.01 && sc[3 * j + 1] > Ninter[k])) {
                    neg.push_back(Kept{nb[3 * j], nb[3 * j + 1], nb[3 * j + 2], c, sc[3 * j + 2], sc[3 * j + 1]});
                    order.set(neg.size() - 1, c / seed_comp);
                    J_out[k] = 1;
                }
            }
        }
        J_out[lin(x, y, z)] = 2;
        if (neg.empty()) break;  // :89-91
        // :93-96 -- the first maximum of C / seed_comp
        const std::pair<double, size_t> fm = order.first_max(neg.size());
        const size_t index = fm.second;
        const double best = std::isnan(fm.first) ? fm.first : neg[index].c / seed_comp;
        ++reg_size;
        if (!(best > 1.0 - drop_off && reg_size < n_mask - 1)) break;  // :98, :121-123
        // :99-119 -- move to the kept voxel; it takes the last kept voxel's place in the list
        const Kept e = neg[index];
        csum += e.c;
        cpos[0] += e.c * e.x;
        cpos[1] += e.c * e.y;
        cpos[2] += e.c * e.z;
        const int64_t k = lin(e.x, e.y, e.z);
        C_out[k] = e.c;
        D_out[k] = e.d;
        N_out[k] = e.n;
        x = e.x;
        y = e.y;
        z = e.z;
        neg[index] = neg.back();
        order.set(index, neg[index].c / seed_comp);
        order.clear(neg.size() - 1);
        neg.pop_back();
    }

    // :127-137 -- the grown voxels (J > 1) in find() order, and the weighted centre
    int64_t count = 0;
    for (int64_t i = 0; i < nvox; ++i) {
        const bool grown = J_out[i] > 1;
        J_out[i] = grown ? 1 : 0;
        if (grown) {
            if (count < idx_cap) idx_out[count] = i + 1;  // 1-based linear index
            ++count;
        }
    }
    *n_idx = count;
    const double center1[3] = {cpos[0] / csum, cpos[1] / csum, cpos[2] / csum};
    const double dx = center1[0] - center0[0], dy = center1[1] - center0[1], dz = center1[2] - center0[2];
    const double lim = maxD > maxD / 10000.0 * (double)count ? maxD : maxD / 10000.0 * (double)count;
    if (std::sqrt(dx * dx + dy * dy + dz * dz) > lim) {
        for (int i = 0; i < 3; ++i) center[i] = mround(center1[i]);
        *replace_center = 1;
    } else {
        for (int i = 0; i < 3; ++i) center[i] = center0[i];
        *replace_center = 0;
    }
    return count > idx_cap ? GRC_ECAPACITY : GRC_OK;
}
