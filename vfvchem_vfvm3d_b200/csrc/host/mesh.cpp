// Jittered-cube mesh generator, exact Bowyer-Watson Delaunay and the Voronoi dual.
//
// This is one-time CPU set-up that produces the inputs of the device assembly kernels.
// Reference behaviour restated here:
//   * delaunay():   src/base/delaunay.rs:6-170 (super-tetrahedron, Morton insertion order,
//                   visibility walk, in-sphere cavity grown until star-shaped, exact predicates);
//   * build_dual(): src/base/geom_tet.rs:101-293 (boundary faces, Voronoi face pieces, sorted
//                   edge list, control-volume volumes and skews, boundary sub-faces, least-squares
//                   gradient weights). Step 6 (pressure-gradient coefficients) is not needed by the
//                   heat path and is not built here.
// The geometric formulas (circumcentres, face pieces, sub-faces) are the reference's, evaluated
// in the same operation order so that results agree to round-off; the data structures are not.
#include "mesh.hpp"

#include <algorithm>
#include <array>
#include <climits>
#include <cmath>
#include <cstring>
#include <memory>
#include <numeric>

namespace vfv {
namespace {

// ---------------------------------------------------------------- random numbers
struct SplitMix64 {  // Steele, Lea & Flood 2014 (public-domain reference constants)
    uint64_t s;
    uint64_t next() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ULL);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
        return z ^ (z >> 31);
    }
    double uniform() { return (double)(next() >> 11) * 0x1.0p-53; }
};

inline double quantize(double x) { return std::nearbyint(std::ldexp(x, kQuantBits)) * std::ldexp(1.0, -kQuantBits); }

// ---------------------------------------------------------------- exact predicates
struct IP { int64_t x, y, z; };
typedef __int128 i128;

// det[a-d; b-d; c-d]; > 0 when d lies below the plane of a, b, c seen counterclockwise from above
inline i128 orient_i(const IP& a, const IP& b, const IP& c, const IP& d) {
    const i128 ax = a.x - d.x, ay = a.y - d.y, az = a.z - d.z;
    const i128 bx = b.x - d.x, by = b.y - d.y, bz = b.z - d.z;
    const i128 cx = c.x - d.x, cy = c.y - d.y, cz = c.z - d.z;
    return ax * (by * cz - bz * cy) - ay * (bx * cz - bz * cx) + az * (bx * cy - by * cx);
}

inline i128 det3(i128 ax, i128 ay, i128 az, i128 bx, i128 by, i128 bz, i128 cx, i128 cy, i128 cz) {
    return ax * (by * cz - bz * cy) - ay * (bx * cz - bz * cx) + az * (bx * cy - by * cx);
}

// > 0 when e is strictly inside the sphere through a, b, c, d (a, b, c, d positively oriented).
// Laplace expansion of the 4x4 lifted determinant along the lifted column; magnitudes stay below
// 2^118 for coordinates within 20 * 2^18 of each other.
inline i128 insphere_i(const IP& a, const IP& b, const IP& c, const IP& d, const IP& e) {
    const i128 ax = a.x - e.x, ay = a.y - e.y, az = a.z - e.z;
    const i128 bx = b.x - e.x, by = b.y - e.y, bz = b.z - e.z;
    const i128 cx = c.x - e.x, cy = c.y - e.y, cz = c.z - e.z;
    const i128 dx = d.x - e.x, dy = d.y - e.y, dz = d.z - e.z;
    const i128 la = ax * ax + ay * ay + az * az;
    const i128 lb = bx * bx + by * by + bz * bz;
    const i128 lc = cx * cx + cy * cy + cz * cz;
    const i128 ld = dx * dx + dy * dy + dz * dz;
    const i128 m_bcd = det3(bx, by, bz, cx, cy, cz, dx, dy, dz);
    const i128 m_acd = det3(ax, ay, az, cx, cy, cz, dx, dy, dz);
    const i128 m_abd = det3(ax, ay, az, bx, by, bz, dx, dy, dz);
    const i128 m_abc = det3(ax, ay, az, bx, by, bz, cx, cy, cz);
    // cofactor expansion of det[a-e, |a-e|^2; ...; d-e, |d-e|^2] along the lifted column
    return lb * m_acd - la * m_bcd + ld * m_abc - lc * m_abd;
}

// Floating-point filters of the two predicates: the same determinant in double with a bound on its
// rounding error, |fl(det) - det| <= c eps * permanent (c is at most about 12 for these expression
// trees; 1e-14 ~ 90 eps leaves a wide margin). Outside the bound the sign is certain; inside it the
// exact 128-bit evaluation decides, so every sign equals the exact one.
inline int orient_sgn(const IP& a, const IP& b, const IP& c, const IP& d) {
    const double ax = (double)(a.x - d.x), ay = (double)(a.y - d.y), az = (double)(a.z - d.z);
    const double bx = (double)(b.x - d.x), by = (double)(b.y - d.y), bz = (double)(b.z - d.z);
    const double cx = (double)(c.x - d.x), cy = (double)(c.y - d.y), cz = (double)(c.z - d.z);
    const double det = ax * (by * cz - bz * cy) - ay * (bx * cz - bz * cx) + az * (bx * cy - by * cx);
    const double perm = std::fabs(ax) * (std::fabs(by * cz) + std::fabs(bz * cy)) + std::fabs(ay) * (std::fabs(bx * cz) + std::fabs(bz * cx)) +
                        std::fabs(az) * (std::fabs(bx * cy) + std::fabs(by * cx));
    const double bound = 1e-14 * perm;
    if (det > bound) return 1;
    if (det < -bound) return -1;
    const i128 e = orient_i(a, b, c, d);
    return (e > 0) - (e < 0);
}

inline int insphere_sgn(const IP& a, const IP& b, const IP& c, const IP& d, const IP& e) {
    const double ax = (double)(a.x - e.x), ay = (double)(a.y - e.y), az = (double)(a.z - e.z);
    const double bx = (double)(b.x - e.x), by = (double)(b.y - e.y), bz = (double)(b.z - e.z);
    const double cx = (double)(c.x - e.x), cy = (double)(c.y - e.y), cz = (double)(c.z - e.z);
    const double dx = (double)(d.x - e.x), dy = (double)(d.y - e.y), dz = (double)(d.z - e.z);
    const double la = ax * ax + ay * ay + az * az, lb = bx * bx + by * by + bz * bz;
    const double lc = cx * cx + cy * cy + cz * cz, ld = dx * dx + dy * dy + dz * dz;
    auto det3d = [](double px, double py, double pz, double qx, double qy, double qz, double rx, double ry, double rz, double& perm) {
        perm = std::fabs(px) * (std::fabs(qy * rz) + std::fabs(qz * ry)) + std::fabs(py) * (std::fabs(qx * rz) + std::fabs(qz * rx)) +
               std::fabs(pz) * (std::fabs(qx * ry) + std::fabs(qy * rx));
        return px * (qy * rz - qz * ry) - py * (qx * rz - qz * rx) + pz * (qx * ry - qy * rx);
    };
    double p_bcd, p_acd, p_abd, p_abc;
    const double m_bcd = det3d(bx, by, bz, cx, cy, cz, dx, dy, dz, p_bcd);
    const double m_acd = det3d(ax, ay, az, cx, cy, cz, dx, dy, dz, p_acd);
    const double m_abd = det3d(ax, ay, az, bx, by, bz, dx, dy, dz, p_abd);
    const double m_abc = det3d(ax, ay, az, bx, by, bz, cx, cy, cz, p_abc);
    const double det = lb * m_acd - la * m_bcd + ld * m_abc - lc * m_abd;
    const double perm = lb * p_acd + la * p_bcd + ld * p_abc + lc * p_abd;
    const double bound = 1e-14 * perm;
    if (det > bound) return 1;
    if (det < -bound) return -1;
    const i128 x = insphere_i(a, b, c, d, e);
    return (x > 0) - (x < 0);
}

inline IP to_ip(const double* p) {
    return IP{(int64_t)std::llround(std::ldexp(p[0], kQuantBits)), (int64_t)std::llround(std::ldexp(p[1], kQuantBits)),
              (int64_t)std::llround(std::ldexp(p[2], kQuantBits))};
}

inline int sgn(i128 v) { return (v > 0) - (v < 0); }

// ---------------------------------------------------------------- vector helpers (geom formulas)
struct V3 { double x, y, z; };
inline V3 add3(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 sub3(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 scale3(double s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
inline double dot3(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross3(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline double len3(V3 a) { return std::sqrt(dot3(a, a)); }

// centre of the circle through a, b, c (delaunay.rs:207-214)
inline V3 circumcircle3(V3 a, V3 b, V3 c) {
    const V3 u = sub3(b, a), v = sub3(c, a);
    const V3 w = cross3(u, v);
    const V3 num = add3(scale3(dot3(u, u), cross3(v, w)), scale3(dot3(v, v), cross3(w, u)));
    return add3(a, scale3(0.5 / dot3(w, w), num));
}

// centre of the sphere through a, b, c, d (delaunay.rs:216-221)
inline V3 circumsphere3(V3 a, V3 b, V3 c, V3 d) {
    const V3 u = sub3(b, a), v = sub3(c, a), w = sub3(d, a);
    const V3 num = add3(add3(scale3(dot3(u, u), cross3(v, w)), scale3(dot3(v, v), cross3(w, u))), scale3(dot3(w, w), cross3(u, v)));
    return add3(a, scale3(0.5 / dot3(u, cross3(v, w)), num));
}

// ---------------------------------------------------------------- exact predicates on doubles
// For vertices off the 2^-18 lattice. A double is an integer times a power of two, so the
// coordinates of one predicate call are exact integers at their smallest exponent; the sign of the
// same determinant as orient_i / insphere_i is then computed on sign-magnitude integers (32-bit
// limbs, schoolbook products). Scaling by a power of two keeps the sign.
struct DP { double x, y, z; };

struct BigInt {
    std::vector<uint32_t> mag;  // little-endian limbs, no leading zero limb
    int sign = 0;               // -1, 0, 1
};

int cmp_mag(const std::vector<uint32_t>& a, const std::vector<uint32_t>& b) {
    if (a.size() != b.size()) return a.size() < b.size() ? -1 : 1;
    for (size_t i = a.size(); i-- > 0;)
        if (a[i] != b[i]) return a[i] < b[i] ? -1 : 1;
    return 0;
}

void trim(std::vector<uint32_t>& m) {
    while (!m.empty() && m.back() == 0) m.pop_back();
}

std::vector<uint32_t> add_mag(const std::vector<uint32_t>& a, const std::vector<uint32_t>& b) {
    const std::vector<uint32_t>& l = a.size() >= b.size() ? a : b;
    const std::vector<uint32_t>& r = a.size() >= b.size() ? b : a;
    std::vector<uint32_t> o(l.size() + 1);
    uint64_t carry = 0;
    for (size_t i = 0; i < l.size(); ++i) {
        const uint64_t t = (uint64_t)l[i] + (i < r.size() ? r[i] : 0u) + carry;
        o[i] = (uint32_t)t;
        carry = t >> 32;
    }
    o[l.size()] = (uint32_t)carry;
    trim(o);
    return o;
}

std::vector<uint32_t> sub_mag(const std::vector<uint32_t>& a, const std::vector<uint32_t>& b) {  // |a| >= |b|
    std::vector<uint32_t> o(a.size());
    int64_t borrow = 0;
    for (size_t i = 0; i < a.size(); ++i) {
        int64_t t = (int64_t)a[i] - (i < b.size() ? (int64_t)b[i] : 0) - borrow;
        borrow = t < 0;
        if (t < 0) t += (int64_t)1 << 32;
        o[i] = (uint32_t)t;
    }
    trim(o);
    return o;
}

BigInt big_add(const BigInt& a, const BigInt& b) {
    if (a.sign == 0) return b;
    if (b.sign == 0) return a;
    BigInt o;
    if (a.sign == b.sign) {
        o.mag = add_mag(a.mag, b.mag);
        o.sign = a.sign;
        return o;
    }
    const int c = cmp_mag(a.mag, b.mag);
    if (c == 0) return o;
    o.mag = c > 0 ? sub_mag(a.mag, b.mag) : sub_mag(b.mag, a.mag);
    o.sign = c > 0 ? a.sign : b.sign;
    return o;
}

BigInt big_neg(BigInt a) {
    a.sign = -a.sign;
    return a;
}

BigInt big_sub(const BigInt& a, const BigInt& b) { return big_add(a, big_neg(b)); }

BigInt big_mul(const BigInt& a, const BigInt& b) {
    BigInt o;
    if (a.sign == 0 || b.sign == 0) return o;
    std::vector<uint64_t> acc(a.mag.size() + b.mag.size() + 1, 0);
    for (size_t i = 0; i < a.mag.size(); ++i) {
        uint64_t carry = 0;
        for (size_t j = 0; j < b.mag.size(); ++j) {
            const uint64_t t = (uint64_t)a.mag[i] * b.mag[j] + (acc[i + j] & 0xffffffffu) + carry;
            acc[i + j] = t & 0xffffffffu;
            carry = t >> 32;
        }
        size_t k = i + b.mag.size();
        while (carry) {
            const uint64_t t = acc[k] + carry;
            acc[k] = t & 0xffffffffu;
            carry = t >> 32;
            ++k;
        }
    }
    o.mag.resize(acc.size());
    for (size_t i = 0; i < acc.size(); ++i) o.mag[i] = (uint32_t)acc[i];
    trim(o.mag);
    o.sign = a.sign * b.sign;
    return o;
}

// exponent of the lowest mantissa bit of a nonzero finite double (x = M 2^E, M odd or 53-bit)
int low_exp(double x) {
    int e = 0;
    (void)std::frexp(x, &e);
    return e - 53;
}

// x / 2^e0 as an exact integer (x a multiple of 2^e0)
BigInt big_from(double x, int e0) {
    BigInt o;
    if (x == 0.0) return o;
    int e = 0;
    const double f = std::frexp(std::fabs(x), &e);
    const uint64_t m = (uint64_t)std::ldexp(f, 53);  // exact: 53-bit integer
    const int sh = e - 53 - e0;                       // >= 0
    o.mag.assign((size_t)(sh / 32) + 3, 0u);
    const int q = sh / 32, r = sh % 32;
    const unsigned __int128 v = (unsigned __int128)m << r;
    o.mag[(size_t)q] = (uint32_t)v;
    o.mag[(size_t)q + 1] = (uint32_t)(v >> 32);
    o.mag[(size_t)q + 2] = (uint32_t)(v >> 64);
    trim(o.mag);
    o.sign = x < 0 ? -1 : 1;
    return o;
}

// the coordinates of k points as integers at their smallest exponent, relative to the last point
template <int K>
void big_diffs(const DP* const (&p)[K], BigInt (&d)[K - 1][3]) {
    int e0 = INT_MAX;
    for (int i = 0; i < K; ++i)
        for (double x : {p[i]->x, p[i]->y, p[i]->z})
            if (x != 0.0) e0 = std::min(e0, low_exp(x));
    if (e0 == INT_MAX) e0 = 0;
    const BigInt lx = big_from(p[K - 1]->x, e0), ly = big_from(p[K - 1]->y, e0), lz = big_from(p[K - 1]->z, e0);
    for (int i = 0; i < K - 1; ++i) {
        d[i][0] = big_sub(big_from(p[i]->x, e0), lx);
        d[i][1] = big_sub(big_from(p[i]->y, e0), ly);
        d[i][2] = big_sub(big_from(p[i]->z, e0), lz);
    }
}

BigInt big_det3(const BigInt* a, const BigInt* b, const BigInt* c) {
    const BigInt t0 = big_sub(big_mul(b[1], c[2]), big_mul(b[2], c[1]));
    const BigInt t1 = big_sub(big_mul(b[0], c[2]), big_mul(b[2], c[0]));
    const BigInt t2 = big_sub(big_mul(b[0], c[1]), big_mul(b[1], c[0]));
    return big_add(big_sub(big_mul(a[0], t0), big_mul(a[1], t1)), big_mul(a[2], t2));
}

int orient_exact(const DP& a, const DP& b, const DP& c, const DP& d) {
    const DP* const p[4] = {&a, &b, &c, &d};
    BigInt q[3][3];
    big_diffs<4>(p, q);
    return big_det3(q[0], q[1], q[2]).sign;
}

int insphere_exact(const DP& a, const DP& b, const DP& c, const DP& d, const DP& e) {
    const DP* const p[5] = {&a, &b, &c, &d, &e};
    BigInt q[4][3];
    big_diffs<5>(p, q);
    BigInt l[4];
    for (int i = 0; i < 4; ++i) l[i] = big_add(big_add(big_mul(q[i][0], q[i][0]), big_mul(q[i][1], q[i][1])), big_mul(q[i][2], q[i][2]));
    const BigInt m_bcd = big_det3(q[1], q[2], q[3]), m_acd = big_det3(q[0], q[2], q[3]);
    const BigInt m_abd = big_det3(q[0], q[1], q[3]), m_abc = big_det3(q[0], q[1], q[2]);
    // the cofactor expansion of insphere_i
    const BigInt r = big_sub(big_add(big_sub(big_mul(l[1], m_acd), big_mul(l[0], m_bcd)), big_mul(l[3], m_abc)), big_mul(l[2], m_abd));
    return r.sign;
}

// Filtered predicates on doubles: the determinant in double from rounded differences. The bound
// 1e-14 * permanent (~45 eps) covers the rounding of the differences as well (Shewchuk 1997 bounds
// this evaluation order by 7 eps for orientation and 16 eps for the in-sphere test); a permanent
// small enough for underflow to matter also goes to the exact evaluation.
constexpr double kTinyPermanent = 1e-250;

inline int orient_sgn(const DP& a, const DP& b, const DP& c, const DP& d) {
    const double ax = a.x - d.x, ay = a.y - d.y, az = a.z - d.z;
    const double bx = b.x - d.x, by = b.y - d.y, bz = b.z - d.z;
    const double cx = c.x - d.x, cy = c.y - d.y, cz = c.z - d.z;
    const double det = ax * (by * cz - bz * cy) - ay * (bx * cz - bz * cx) + az * (bx * cy - by * cx);
    const double perm = std::fabs(ax) * (std::fabs(by * cz) + std::fabs(bz * cy)) + std::fabs(ay) * (std::fabs(bx * cz) + std::fabs(bz * cx)) +
                        std::fabs(az) * (std::fabs(bx * cy) + std::fabs(by * cx));
    const double bound = 1e-14 * perm;
    if (perm > kTinyPermanent) {
        if (det > bound) return 1;
        if (det < -bound) return -1;
    }
    return orient_exact(a, b, c, d);
}

inline int insphere_sgn(const DP& a, const DP& b, const DP& c, const DP& d, const DP& e) {
    const double ax = a.x - e.x, ay = a.y - e.y, az = a.z - e.z;
    const double bx = b.x - e.x, by = b.y - e.y, bz = b.z - e.z;
    const double cx = c.x - e.x, cy = c.y - e.y, cz = c.z - e.z;
    const double dx = d.x - e.x, dy = d.y - e.y, dz = d.z - e.z;
    const double la = ax * ax + ay * ay + az * az, lb = bx * bx + by * by + bz * bz;
    const double lc = cx * cx + cy * cy + cz * cz, ld = dx * dx + dy * dy + dz * dz;
    auto det3d = [](double px, double py, double pz, double qx, double qy, double qz, double rx, double ry, double rz, double& perm) {
        perm = std::fabs(px) * (std::fabs(qy * rz) + std::fabs(qz * ry)) + std::fabs(py) * (std::fabs(qx * rz) + std::fabs(qz * rx)) +
               std::fabs(pz) * (std::fabs(qx * ry) + std::fabs(qy * rx));
        return px * (qy * rz - qz * ry) - py * (qx * rz - qz * rx) + pz * (qx * ry - qy * rx);
    };
    double p_bcd, p_acd, p_abd, p_abc;
    const double m_bcd = det3d(bx, by, bz, cx, cy, cz, dx, dy, dz, p_bcd);
    const double m_acd = det3d(ax, ay, az, cx, cy, cz, dx, dy, dz, p_acd);
    const double m_abd = det3d(ax, ay, az, bx, by, bz, dx, dy, dz, p_abd);
    const double m_abc = det3d(ax, ay, az, bx, by, bz, cx, cy, cz, p_abc);
    const double det = lb * m_acd - la * m_bcd + ld * m_abc - lc * m_abd;
    const double perm = lb * p_acd + la * p_bcd + ld * p_abc + lc * p_abd;
    const double bound = 1e-14 * perm;
    if (perm > kTinyPermanent) {
        if (det > bound) return 1;
        if (det < -bound) return -1;
    }
    return insphere_exact(a, b, c, d, e);
}

inline bool same_pt(const IP& a, const IP& b) { return a.x == b.x && a.y == b.y && a.z == b.z; }
inline bool same_pt(const DP& a, const DP& b) { return a.x == b.x && a.y == b.y && a.z == b.z; }

inline uint64_t spread3(uint64_t v) {  // 21 bits -> every third bit
    v &= 0x1fffffULL;
    v = (v | (v << 32)) & 0x1f00000000ffffULL;
    v = (v | (v << 16)) & 0x1f0000ff0000ffULL;
    v = (v | (v << 8)) & 0x100f00f00f00f00fULL;
    v = (v | (v << 4)) & 0x10c30c30c30c30c3ULL;
    v = (v | (v << 2)) & 0x1249249249249249ULL;
    return v;
}

}  // namespace


// ---------------------------------------------------------------- mesh generator
Mesh make_jitter_cube(int n, uint64_t seed, double jitter) {
    Mesh m;
    if (n < 3) return m;
    const double h = 1.0 / (double)(n - 1);
    SplitMix64 rng{seed};
    std::vector<double> pts;
    std::vector<double> nds[NUM_BND];
    for (int k = 0; k < n; ++k)
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) {
                const double u0 = rng.uniform(), u1 = rng.uniform(), u2 = rng.uniform();
                const bool fx = (i == 0 || i == n - 1), fy = (j == 0 || j == n - 1), fz = (k == 0 || k == n - 1);
                double x = (double)i / (double)(n - 1), y = (double)j / (double)(n - 1), z = (double)k / (double)(n - 1);
                if (!fx) x += (2.0 * u0 - 1.0) * jitter * h;
                if (!fy) y += (2.0 * u1 - 1.0) * jitter * h;
                if (!fz) z += (2.0 * u2 - 1.0) * jitter * h;
                x = quantize(x);
                y = quantize(y);
                z = quantize(z);
                if (!fx && !fy && !fz) {
                    pts.insert(pts.end(), {x, y, z});
                } else {
                    const int b = fx ? (i == 0 ? BND_L : BND_R) : fy ? (j == 0 ? BND_F : BND_K) : (k == 0 ? BND_B : BND_T);
                    nds[b].insert(nds[b].end(), {x, y, z});
                }
            }
    m.n_pts = (int64_t)pts.size() / 3;
    m.pos = std::move(pts);
    for (int b = 0; b < NUM_BND; ++b) {
        m.pos.insert(m.pos.end(), nds[b].begin(), nds[b].end());
        m.node_bnd.insert(m.node_bnd.end(), nds[b].size() / 3, b);
    }
    m.n_nds = (int64_t)m.node_bnd.size();
    return m;
}

// ---------------------------------------------------------------- Delaunay
namespace {

// Bowyer-Watson insertion over the points P (the mesh's vertices, then the four super vertices)
// with the exact predicates of their type.
template <typename Pt>
std::string bowyer_watson(Mesh& mesh, const std::vector<Pt>& P, const double lo[3], const double hi[3], double size) {
    const int64_t N = mesh.n_tot();
    std::vector<std::array<int32_t, 4>> tv, ta;
    std::vector<uint8_t> alive, incav;
    std::vector<int32_t> freel;
    tv.reserve(7 * N + 64);
    ta.reserve(7 * N + 64);
    tv.push_back({(int32_t)N, (int32_t)N + 1, (int32_t)N + 2, (int32_t)N + 3});
    if (orient_sgn(P[N], P[N + 1], P[N + 2], P[N + 3]) < 0) std::swap(tv[0][0], tv[0][1]);
    ta.push_back({-1, -1, -1, -1});
    alive.push_back(1);
    incav.push_back(0);

    // insertion order: Morton code of the quantised position, ties by vid
    std::vector<std::pair<uint64_t, int32_t>> order(N);
    for (int64_t v = 0; v < N; ++v) {
        uint64_t q[3];
        for (int c = 0; c < 3; ++c) {
            double t = (mesh.pos[3 * v + c] - lo[c]) / size * 2097151.0;
            q[c] = (uint64_t)std::min(2097151.0, std::max(0.0, t));
        }
        order[v] = {spread3(q[0]) | (spread3(q[1]) << 1) | (spread3(q[2]) << 2), (int32_t)v};
    }
    std::sort(order.begin(), order.end());

    auto tet_pts = [&](int32_t t, Pt q[4]) {
        for (int c = 0; c < 4; ++c) q[c] = P[tv[t][c]];
    };

    std::vector<int32_t> cav;
    struct BF { int32_t t, k; };
    std::vector<BF> bfaces;
    struct EdgeSlot { int64_t key; int32_t t, m; };  // key -1: empty; t -1: no tetrahedron waiting
    std::vector<EdgeSlot> etab;
    std::vector<int32_t> eused;
    std::vector<int32_t> newt;
    int32_t last = 0;
    unsigned turn = 0;
    Pt q[4];
    for (int64_t oi = 0; oi < N; ++oi) {
        const int32_t vid = order[oi].second;
        const Pt p = P[vid];
        // locate by a visibility walk; fall back to a scan if the walk runs long
        int32_t t = last;
        int64_t steps = 0;
        for (;;) {
            if (++steps > 4 * (int64_t)tv.size() + 16) {
                t = -1;
                for (int32_t s = 0; s < (int32_t)tv.size() && t < 0; ++s) {
                    if (!alive[s]) continue;
                    bool in = true;
                    for (int k = 0; k < 4 && in; ++k) {
                        tet_pts(s, q);
                        q[k] = p;
                        in = orient_sgn(q[0], q[1], q[2], q[3]) >= 0;
                    }
                    if (in) t = s;
                }
                if (t < 0) return "delaunay: point location failed";
                break;
            }
            turn = (turn + 1) & 3u;
            bool moved = false;
            for (int l = 0; l < 4; ++l) {
                const int k = (int)((l + turn) & 3u);
                tet_pts(t, q);
                q[k] = p;
                if (orient_sgn(q[0], q[1], q[2], q[3]) < 0) {
                    const int32_t o = ta[t][k];
                    if (o < 0) return "delaunay: point outside the super tetrahedron";
                    t = o;
                    moved = true;
                    break;
                }
            }
            if (!moved) break;
        }
        for (int k = 0; k < 4; ++k)
            if (same_pt(P[tv[t][k]], p)) return "delaunay: duplicate vertex";
        // cavity: tetrahedra whose circumsphere strictly contains p
        cav.clear();
        cav.push_back(t);
        incav[t] = 1;
        bool tie = false;  // p on the circumsphere of a tetrahedron next to the cavity
        for (size_t i = 0; i < cav.size(); ++i) {
            const int32_t c = cav[i];
            for (int k = 0; k < 4; ++k) {
                const int32_t o = ta[c][k];
                if (o < 0 || incav[o]) continue;
                tet_pts(o, q);
                const int sg = insphere_sgn(q[0], q[1], q[2], q[3], p);
                if (sg > 0) {
                    incav[o] = 1;
                    cav.push_back(o);
                } else if (sg == 0) {
                    tie = true;
                }
            }
        }
        // grow until every boundary face sees p with positive orientation (cospherical ties).
        // Without a tie the cavity is already star-shaped: a boundary face joins c (p strictly
        // inside its circumsphere) and o (p strictly outside); the two spheres meet in the face's
        // circle and, the triangulation being Delaunay, o's ball holds c's on o's side of the
        // face's plane, so p lies strictly on c's side and the loop would add nothing.
        for (bool star = !tie; !star;) {
            star = true;
            for (size_t i = 0; i < cav.size(); ++i) {
                const int32_t c = cav[i];
                for (int k = 0; k < 4; ++k) {
                    const int32_t o = ta[c][k];
                    if (o >= 0 && incav[o]) continue;
                    tet_pts(c, q);
                    q[k] = p;
                    if (orient_sgn(q[0], q[1], q[2], q[3]) > 0) continue;
                    if (o < 0) return "delaunay: cavity reaches the super tetrahedron hull";
                    incav[o] = 1;
                    cav.push_back(o);
                    star = false;
                }
            }
        }
        // boundary faces of the cavity, then one new tetrahedron per face
        bfaces.clear();
        for (int32_t c : cav)
            for (int k = 0; k < 4; ++k) {
                const int32_t o = ta[c][k];
                if (o >= 0 && incav[o]) continue;
                bfaces.push_back({c, k});
            }
        newt.resize(bfaces.size());
        for (size_t i = 0; i < bfaces.size(); ++i) {
            if (!freel.empty()) {
                newt[i] = freel.back();
                freel.pop_back();
            } else {
                newt[i] = (int32_t)tv.size();
                tv.push_back({0, 0, 0, 0});
                ta.push_back({-1, -1, -1, -1});
                alive.push_back(0);
                incav.push_back(0);
            }
        }
        // edges of the cavity boundary in a hash table sized for load <= 1/4
        int ebits = 4;
        while ((size_t{1} << ebits) < 6 * bfaces.size()) ++ebits;
        const uint64_t emask = (uint64_t{1} << ebits) - 1;
        if (etab.size() < (size_t{1} << ebits)) etab.assign(size_t{1} << ebits, EdgeSlot{-1, -1, 0});
        int64_t n_open = 0;
        for (size_t i = 0; i < bfaces.size(); ++i) {
            const int32_t c = bfaces[i].t, k = bfaces[i].k, nt = newt[i];
            std::array<int32_t, 4> nv = tv[c];
            nv[k] = vid;
            tv[nt] = nv;
            ta[nt] = {-1, -1, -1, -1};
            alive[nt] = 1;
            const int32_t o = ta[c][k];
            ta[nt][k] = o;
            if (o >= 0)
                for (int mm = 0; mm < 4; ++mm)
                    if (ta[o][mm] == c) {
                        ta[o][mm] = nt;
                        break;
                    }
            for (int mm = 0; mm < 4; ++mm) {
                if (mm == k) continue;
                int32_t e2[2], ne = 0;
                for (int l = 0; l < 4; ++l)
                    if (l != k && l != mm) e2[ne++] = nv[l];
                const int64_t key = ((int64_t)std::min(e2[0], e2[1]) << 32) | (int64_t)std::max(e2[0], e2[1]);
                uint64_t h = ((uint64_t)key * 0x9E3779B97F4A7C15ULL) >> (64 - ebits);
                while (etab[h].key != key && etab[h].key != -1) h = (h + 1) & emask;
                EdgeSlot& sl = etab[h];
                if (sl.key == -1) {
                    sl.key = key;
                    eused.push_back((int32_t)h);
                }
                if (sl.t >= 0) {  // the other new tetrahedron on this edge
                    ta[nt][mm] = sl.t;
                    ta[sl.t][sl.m] = nt;
                    sl.t = -1;
                    --n_open;
                } else {
                    sl.t = nt;
                    sl.m = mm;
                    ++n_open;
                }
            }
        }
        for (int32_t h : eused) etab[h] = EdgeSlot{-1, -1, 0};
        eused.clear();
        if (n_open != 0) return "delaunay: cavity boundary is not closed";
        for (int32_t c : cav) {
            alive[c] = 0;
            incav[c] = 0;
            freel.push_back(c);
        }
        last = newt.back();
    }

    mesh.tets.clear();
    double vol = 0.0;
    for (size_t t = 0; t < tv.size(); ++t) {
        if (!alive[t]) continue;
        const auto& v = tv[t];
        if (v[0] >= N || v[1] >= N || v[2] >= N || v[3] >= N) continue;
        mesh.tets.insert(mesh.tets.end(), v.begin(), v.end());
        const double* a = &mesh.pos[3 * v[0]];
        const double* b = &mesh.pos[3 * v[1]];
        const double* c = &mesh.pos[3 * v[2]];
        const double* d = &mesh.pos[3 * v[3]];
        const V3 ad{a[0] - d[0], a[1] - d[1], a[2] - d[2]}, bd{b[0] - d[0], b[1] - d[1], b[2] - d[2]},
            cd{c[0] - d[0], c[1] - d[1], c[2] - d[2]};
        vol += dot3(ad, cross3(bd, cd)) / 6.0;
    }
    if (mesh.tets.empty()) return "delaunay: no tetrahedra";
    const double hull = (hi[0] - lo[0]) * (hi[1] - lo[1]) * (hi[2] - lo[2]);
    if (std::fabs(vol - hull) > 1e-9 * hull) return "delaunay: tetrahedra do not fill the bounding box (hull is not a box)";
    return "";
}

}  // namespace

// Vertices on the 2^-18 lattice within the range of the 128-bit predicates (the generated cubes)
// take the integer predicates; any other finite coordinates the filtered double predicates with an
// exact fallback. Both give the exact signs, so the same input gives the same tetrahedra.
std::string delaunay(Mesh& mesh) {
    const int64_t N = mesh.n_tot();
    if (N < 4) return "delaunay: fewer than four vertices";
    if (N > (int64_t)0x7ffffff0) return "delaunay: too many vertices for 32-bit ids";
    constexpr double kMaxBoxLattice = 1.75;  // the integer predicates' range (with the super vertices)
    constexpr double kMaxCoord = 1e50;       // double predicates: products of degree 5 stay finite
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    bool lattice = true;
    for (int64_t v = 0; v < N; ++v)
        for (int c = 0; c < 3; ++c) {
            const double x = mesh.pos[3 * v + c];
            if (!(std::fabs(x) <= kMaxCoord)) return "delaunay: coordinates must be finite and within 1e50 in magnitude";
            lo[c] = std::min(lo[c], x);
            hi[c] = std::max(hi[c], x);
            const double q = std::ldexp(x, kQuantBits);
            if (q != std::nearbyint(q) || !(std::fabs(x) < 8.0)) lattice = false;
        }
    for (int c = 0; c < 3; ++c)
        if (hi[c] - lo[c] > kMaxBoxLattice) lattice = false;
    const double size = std::max({hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2], 1e-300});
    const double cen[3] = {0.5 * (lo[0] + hi[0]), 0.5 * (lo[1] + hi[1]), 0.5 * (lo[2] + hi[2])};
    const double dirs[4][3] = {{1, 1, 1}, {1, -1, -1}, {-1, 1, -1}, {-1, -1, 1}};
    double sup[4][3];
    for (int s = 0; s < 4; ++s)
        for (int c = 0; c < 3; ++c) sup[s][c] = cen[c] + 10.0 * size * dirs[s][c];
    if (lattice) {
        std::vector<IP> P(N + 4);
        for (int64_t v = 0; v < N; ++v) P[v] = to_ip(&mesh.pos[3 * v]);
        for (int s = 0; s < 4; ++s) P[N + s] = to_ip(sup[s]);
        return bowyer_watson(mesh, P, lo, hi, size);
    }
    std::vector<DP> P(N + 4);
    for (int64_t v = 0; v < N; ++v) P[v] = DP{mesh.pos[3 * v], mesh.pos[3 * v + 1], mesh.pos[3 * v + 2]};
    for (int s = 0; s < 4; ++s) P[N + s] = DP{sup[s][0], sup[s][1], sup[s][2]};
    return bowyer_watson(mesh, P, lo, hi, size);
}

// ---------------------------------------------------------------- Voronoi dual
namespace {

constexpr int kEdgeEnds[6][2] = {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {1, 3}, {2, 3}};

// The two Voronoi face pieces that tetrahedron tv (circumcentre c_t) contributes to its local edge
// e (geom_tet.rs:122-171): per side, the area of the triangle (edge midpoint, circumcentre of the
// face towards that side, c_t) signed along the normal pointing away from the other side, and the
// triangle's centroid.
inline void face_pieces(const Mesh& mesh, const int32_t* tv, V3 c_t, int e, double area[2], V3 cent[2]) {
    auto P = [&](int64_t v) { return V3{mesh.pos[3 * v], mesh.pos[3 * v + 1], mesh.pos[3 * v + 2]}; };
    const int li = kEdgeEnds[e][0], lj = kEdgeEnds[e][1];
    int oth[2], no = 0;
    for (int l = 0; l < 4; ++l)
        if (l != li && l != lj) oth[no++] = l;
    const V3 pi = P(tv[li]), pj = P(tv[lj]);
    const double dist = len3(sub3(pj, pi));
    const V3 ee = scale3(1.0 / dist, sub3(pj, pi));
    const V3 m = scale3(0.5, add3(pi, pj));
    for (int side = 0; side < 2; ++side) {
        const V3 pa = P(tv[oth[side]]), pb = P(tv[oth[1 - side]]);
        const V3 c_f = circumcircle3(pi, pj, pa);
        V3 u = sub3(sub3(pa, m), scale3(dot3(sub3(pa, m), ee), ee));
        u = scale3(1.0 / len3(u), u);
        V3 n = cross3(ee, u);
        if (dot3(sub3(pb, m), n) < 0.0) n = scale3(-1.0, n);
        const double s1 = dot3(sub3(c_f, m), u);
        const double s2 = dot3(sub3(c_t, c_f), n);
        area[side] = 0.5 * s1 * s2;
        cent[side] = scale3(1.0 / 3.0, add3(m, add3(c_f, c_t)));
    }
}

}  // namespace

// Boundary sub-faces (geom_tet.rs:208-259) of the faces flagged in bface[4 t + k] (the face
// opposite local vertex k of tetrahedron t is a boundary face), visited in (tetrahedron, face)
// order; fills d.bnd_* and d.bnd_sum. Returns "" on success.
std::string boundary_subfaces(const Mesh& mesh, const std::vector<uint8_t>& bface, Dual& d) {
    const int64_t N = mesh.n_tot(), T = mesh.n_tet();
    const int32_t* tet = mesh.tets.data();
    auto P = [&](int64_t v) { return V3{mesh.pos[3 * v], mesh.pos[3 * v + 1], mesh.pos[3 * v + 2]}; };
    static const int FO[4][3] = {{1, 3, 2}, {0, 2, 3}, {0, 3, 1}, {0, 1, 2}};  // counterclockwise from outside
    std::vector<int32_t> surf;
    for (int64_t t = 0; t < T; ++t)
        for (int k = 0; k < 4; ++k)
            if (bface[4 * t + k]) surf.insert(surf.end(), {tet[4 * t + FO[k][0]], tet[4 * t + FO[k][1]], tet[4 * t + FO[k][2]]});
    for (int32_t v : surf)
        if (v < mesh.n_pts) return "dual: a boundary face joins an interior point";
    // ---- boundary sub-faces (geom_tet.rs:208-259)
    const int64_t S = (int64_t)surf.size() / 3;
    d.bnd_ptr.assign(N + 1, 0);
    for (int64_t s = 0; s < S; ++s)
        for (int l = 0; l < 3; ++l) d.bnd_ptr[surf[3 * s + l] + 1]++;
    for (int64_t v = 0; v < N; ++v) d.bnd_ptr[v + 1] += d.bnd_ptr[v];
    const int64_t B = d.bnd_ptr[N];
    d.bnd_j.assign(B, 0);
    d.bnd_k.assign(B, 0);
    d.bnd_area.assign(B, 0.0);
    d.bnd_norm.assign(3 * B, 0.0);
    d.bnd_wgt.assign(3 * B, 0.0);
    d.bnd_sum.assign(N, 0.0);
    std::vector<int64_t> bcur(d.bnd_ptr.begin(), d.bnd_ptr.end() - 1);
    for (int64_t s = 0; s < S; ++s) {
        const int32_t* tt = &surf[3 * s];
        const V3 p0 = P(tt[0]), p1 = P(tt[1]), p2 = P(tt[2]);
        V3 nrm = cross3(sub3(p1, p0), sub3(p2, p0));
        nrm = scale3(1.0 / len3(nrm), nrm);
        const V3 c = circumcircle3(p0, p1, p2);
        const double sq[3] = {dot3(sub3(p2, p1), sub3(p2, p1)), dot3(sub3(p0, p2), sub3(p0, p2)), dot3(sub3(p1, p0), sub3(p1, p0))};
        const double lraw[3] = {sq[0] * (sq[1] + sq[2] - sq[0]), sq[1] * (sq[2] + sq[0] - sq[1]), sq[2] * (sq[0] + sq[1] - sq[2])};
        const double lsum = lraw[0] + lraw[1] + lraw[2];
        const double lam[3] = {lraw[0] / lsum, lraw[1] / lsum, lraw[2] / lsum};
        for (int loc = 0; loc < 3; ++loc) {
            const int32_t vi = tt[loc], vj = tt[(loc + 1) % 3], vk = tt[(loc + 2) % 3];
            const V3 pi = P(vi), pj = P(vj), pk = P(vk);
            double ar[2];
            for (int side = 0; side < 2; ++side) {
                const V3 pa = side == 0 ? pj : pk, pb = side == 0 ? pk : pj;
                const V3 m = scale3(0.5, add3(pi, pa));
                const V3 e = sub3(pa, pi);
                const double len = len3(e);
                const V3 u = sub3(sub3(pb, m), scale3(dot3(sub3(pb, m), e) / (len * len), e));
                ar[side] = 0.25 * len * dot3(sub3(c, m), scale3(1.0 / len3(u), u));
            }
            const double asum = ar[0] + ar[1];
            const double l0 = lam[loc], l1 = lam[(loc + 1) % 3], l2 = lam[(loc + 2) % 3];
            const V3 cj{(1.5 + l0) / 3.0, (0.5 + l1) / 3.0, l2 / 3.0};
            const V3 ck{(1.5 + l0) / 3.0, l1 / 3.0, (0.5 + l2) / 3.0};
            const V3 w = (std::fabs(asum) > 1e-12 * len3(sub3(pj, pi)) * len3(sub3(pk, pi)))
                             ? scale3(1.0 / asum, add3(scale3(ar[0], cj), scale3(ar[1], ck)))
                             : V3{1.0, 0.0, 0.0};
            const int64_t ib = bcur[vi]++;
            d.bnd_sum[vi] += asum;
            d.bnd_j[ib] = vj;
            d.bnd_k[ib] = vk;
            d.bnd_area[ib] = asum;
            d.bnd_norm[ib] = nrm.x;
            d.bnd_norm[B + ib] = nrm.y;
            d.bnd_norm[2 * B + ib] = nrm.z;
            d.bnd_wgt[ib] = w.x;
            d.bnd_wgt[B + ib] = w.y;
            d.bnd_wgt[2 * B + ib] = w.z;
        }
    }

    return "";
}

// Every step is a data-parallel pass over tetrahedra, vertices or edges. Each sum runs in the
// order of the serial tetrahedron loop of the reference (tetrahedron, then local edge, then side),
// so the result does not depend on the thread count.
std::string build_dual(const Mesh& mesh, Dual& d, double piece_store_bytes) {
    const int64_t N = mesh.n_tot(), T = mesh.n_tet();
    const int32_t* tet = mesh.tets.data();
    auto P = [&](int64_t v) { return V3{mesh.pos[3 * v], mesh.pos[3 * v + 1], mesh.pos[3 * v + 2]}; };
    if (N >= (int64_t)INT32_MAX || T >= (int64_t)INT32_MAX) return "dual: mesh too large for 32-bit indices";
    for (int64_t i = 0; i < 4 * T; ++i)
        if (tet[i] < 0 || tet[i] >= N) return "dual: tetrahedron vertex out of range";

    // ---- vertex -> tetrahedra, ascending tetrahedron index per vertex
    std::vector<int64_t> vt_ptr(N + 1, 0);
    for (int64_t i = 0; i < 4 * T; ++i) vt_ptr[tet[i] + 1]++;
    for (int64_t v = 0; v < N; ++v) vt_ptr[v + 1] += vt_ptr[v];
    std::vector<int32_t> vt_idx(4 * T);
    {
        std::vector<int64_t> cur(vt_ptr.begin(), vt_ptr.end() - 1);
        for (int64_t t = 0; t < T; ++t)
            for (int k = 0; k < 4; ++k) vt_idx[cur[tet[4 * t + k]]++] = (int32_t)t;
    }

    // ---- neighbour CSR (geom_tet.rs:173-206): the sorted edge list read per vertex is its
    //      neighbours in ascending order, so the lists come from the incident tetrahedra directly
    d = Dual();
    d.n_tot = N;
    d.n_pts = mesh.n_pts;
    // distinct vertices of v's tetrahedra: stamp[u] == v marks u as taken (one stamp array per
    // thread and pass; a vertex is handled by one thread), then the few distinct ones are sorted
    auto gather = [&](int64_t v, std::vector<int32_t>& buf, std::vector<int32_t>& stamp) {
        buf.clear();
        for (int64_t q = vt_ptr[v]; q < vt_ptr[v + 1]; ++q) {
            const int32_t* tv = &tet[4 * (int64_t)vt_idx[q]];
            for (int k = 0; k < 4; ++k) {
                const int32_t u = tv[k];
                if (u != v && stamp[u] != (int32_t)v) {
                    stamp[u] = (int32_t)v;
                    buf.push_back(u);
                }
            }
        }
        std::sort(buf.begin(), buf.end());
    };
    d.nbr_ptr.assign(N + 1, 0);
#pragma omp parallel
    {
        std::vector<int32_t> buf, stamp(N, -1);
#pragma omp for schedule(dynamic, 1024)
        for (int64_t v = 0; v < N; ++v) {
            gather(v, buf, stamp);
            d.nbr_ptr[v + 1] = (int64_t)buf.size();
        }
    }
    for (int64_t v = 0; v < N; ++v) d.nbr_ptr[v + 1] += d.nbr_ptr[v];
    const int64_t D = d.nbr_ptr[N];
    d.n_dir = D;
    d.nbr_idx.assign(D, 0);
#pragma omp parallel
    {
        std::vector<int32_t> buf, stamp(N, -1);
#pragma omp for schedule(dynamic, 1024)
        for (int64_t v = 0; v < N; ++v) {
            gather(v, buf, stamp);
            std::copy(buf.begin(), buf.end(), d.nbr_idx.begin() + d.nbr_ptr[v]);
        }
    }
    auto nbr_pos = [&](int64_t v, int32_t n) {  // position of n in v's list (present by construction)
        return (int64_t)(std::lower_bound(d.nbr_idx.begin() + d.nbr_ptr[v], d.nbr_idx.begin() + d.nbr_ptr[v + 1], n) - d.nbr_idx.begin());
    };

    // ---- Voronoi face pieces of every tetrahedron edge (geom_tet.rs:122-171): stored (384 bytes
    //      per tetrahedron) while that fits the budget, else recomputed where needed from the
    //      stored circumcentres (24 bytes per tetrahedron; the same function, so the same bits)
    const bool store = (double)T * 48.0 * sizeof(double) <= piece_store_bytes;
    // every entry is written below; left uninitialised so that the parallel loop first-touches it
    std::unique_ptr<double[]> pc_area, pc_cent, ctc;
    if (store) {
        pc_area.reset(new double[12 * T]);
        pc_cent.reset(new double[36 * T]);
    } else {
        ctc.reset(new double[3 * T]);
    }
#pragma omp parallel for schedule(static)
    for (int64_t t = 0; t < T; ++t) {
        const int32_t* tv = &tet[4 * t];
        const V3 c_t = circumsphere3(P(tv[0]), P(tv[1]), P(tv[2]), P(tv[3]));
        if (!store) {
            ctc[3 * t] = c_t.x;
            ctc[3 * t + 1] = c_t.y;
            ctc[3 * t + 2] = c_t.z;
            continue;
        }
        for (int e = 0; e < 6; ++e) {
            double a[2];
            V3 c[2];
            face_pieces(mesh, tv, c_t, e, a, c);
            for (int side = 0; side < 2; ++side) {
                const int64_t q = 12 * t + 2 * e + side;
                pc_area[q] = a[side];
                pc_cent[3 * q] = c[side].x;
                pc_cent[3 * q + 1] = c[side].y;
                pc_cent[3 * q + 2] = c[side].z;
            }
        }
    }
    auto pieces = [&](int64_t t, int e, double a[2], V3 c[2]) {
        if (store) {
            for (int side = 0; side < 2; ++side) {
                const int64_t q = 12 * t + 2 * e + side;
                a[side] = pc_area[q];
                c[side] = V3{pc_cent[3 * q], pc_cent[3 * q + 1], pc_cent[3 * q + 2]};
            }
        } else {
            face_pieces(mesh, &tet[4 * t], V3{ctc[3 * t], ctc[3 * t + 1], ctc[3 * t + 2]}, e, a, c);
        }
    };

    // ---- per edge (a, b), a < b: area and skew summed over its tetrahedra in ascending order,
    //      then the data of both directed entries. The tetrahedra of every edge (a, b > a) come
    //      from one scan of a's tetrahedra (ascending, so each edge's list is ascending too).
    //      Boundary faces (geom_tet.rs:101-116: faces of exactly one tetrahedron) are found here
    //      as well: a face whose two smallest vertices are a < b and whose third is z > b is a
    //      boundary face when one tetrahedron of edge (a, b) holds z; each face is visited once.
    d.nbr_rev.assign(D, 0);
    d.dist.assign(D, 0.0);
    d.area.assign(D, 0.0);
    d.norm.assign(3 * D, 0.0);
    d.skew.assign(3 * D, 0.0);
    std::vector<uint8_t> bface(4 * T, 0);  // [4 t + k]: face opposite local vertex k is a boundary face
#pragma omp parallel
    {
        std::vector<int32_t> slot(N, 0), cnt, fill, lst;
#pragma omp for schedule(dynamic, 1024)
        for (int64_t a = 0; a < N; ++a) {
            const int64_t u0 = std::upper_bound(d.nbr_idx.begin() + d.nbr_ptr[a], d.nbr_idx.begin() + d.nbr_ptr[a + 1], (int32_t)a) - d.nbr_idx.begin();
            const int64_t up = d.nbr_ptr[a + 1] - u0;  // neighbours above a
            if (up == 0) continue;
            for (int64_t k = 0; k < up; ++k) slot[d.nbr_idx[u0 + k]] = (int32_t)k;
            cnt.assign(up + 1, 0);
            for (int64_t q = vt_ptr[a]; q < vt_ptr[a + 1]; ++q) {
                const int32_t* tv = &tet[4 * (int64_t)vt_idx[q]];
                for (int l = 0; l < 4; ++l)
                    if (tv[l] > a) cnt[slot[tv[l]] + 1]++;
            }
            for (int64_t k = 0; k < up; ++k) cnt[k + 1] += cnt[k];
            fill.assign(cnt.begin(), cnt.end() - 1);
            lst.resize(cnt[up]);
            for (int64_t q = vt_ptr[a]; q < vt_ptr[a + 1]; ++q) {
                const int32_t* tv = &tet[4 * (int64_t)vt_idx[q]];
                for (int l = 0; l < 4; ++l)
                    if (tv[l] > a) lst[fill[slot[tv[l]]]++] = vt_idx[q];
            }
            for (int64_t k = 0; k < up; ++k) {
                const int64_t ia = u0 + k;
                const int32_t b = d.nbr_idx[ia];
                double s_area = 0.0, s_x = 0.0, s_y = 0.0, s_z = 0.0;
                for (int32_t j = cnt[k]; j < cnt[k + 1]; ++j) {
                    const int64_t t = lst[j];
                    const int32_t* tv = &tet[4 * t];
                    int e = 0;
                    while (!((tv[kEdgeEnds[e][0]] == a && tv[kEdgeEnds[e][1]] == b) || (tv[kEdgeEnds[e][0]] == b && tv[kEdgeEnds[e][1]] == a))) ++e;
                    const V3 m = scale3(0.5, add3(P(tv[kEdgeEnds[e][0]]), P(tv[kEdgeEnds[e][1]])));
                    double pa[2];
                    V3 pcen[2];
                    pieces(t, e, pa, pcen);
                    for (int side = 0; side < 2; ++side) {
                        const double area = pa[side];
                        const V3 cent = pcen[side];
                        s_area += area;
                        const V3 sk = scale3(area, sub3(cent, m));
                        s_x += sk.x;
                        s_y += sk.y;
                        s_z += sk.z;
                    }
                    for (int l = 0; l < 4; ++l) {  // faces (a, b, z) with z > b
                        const int32_t z = tv[l];
                        if (z <= b) continue;
                        int holders = 0;
                        for (int32_t j2 = cnt[k]; j2 < cnt[k + 1] && holders < 2; ++j2) {
                            const int32_t* w = &tet[4 * (int64_t)lst[j2]];
                            holders += (w[0] == z) | (w[1] == z) | (w[2] == z) | (w[3] == z);
                        }
                        if (holders == 1) {
                            int opp = 0;  // the local vertex not on the face
                            while (tv[opp] == a || tv[opp] == b || tv[opp] == z) ++opp;
                            bface[4 * t + opp] = 1;
                        }
                    }
                }
                const V3 pa = P(a), pb = P(b);
                const double dist = len3(sub3(pb, pa));
                const V3 nrm = scale3(1.0 / dist, sub3(pb, pa));
                const V3 skew = (std::fabs(s_area) > 1e-12 * dist * dist) ? scale3(1.0 / s_area, V3{s_x, s_y, s_z}) : V3{0.0, 0.0, 0.0};
                const int64_t ib = nbr_pos(b, (int32_t)a);
                d.nbr_rev[ia] = ib;
                d.nbr_rev[ib] = ia;
                d.dist[ia] = d.dist[ib] = dist;
                d.area[ia] = d.area[ib] = s_area;
                const V3 mn = scale3(-1.0, nrm);
                d.norm[ia] = nrm.x;
                d.norm[D + ia] = nrm.y;
                d.norm[2 * D + ia] = nrm.z;
                d.norm[ib] = mn.x;
                d.norm[D + ib] = mn.y;
                d.norm[2 * D + ib] = mn.z;
                d.skew[ia] = d.skew[ib] = skew.x;
                d.skew[D + ia] = d.skew[D + ib] = skew.y;
                d.skew[2 * D + ia] = d.skew[2 * D + ib] = skew.z;
            }
        }
    }

    // ---- per vertex: control volume (faces in neighbour order) and its centroid offset (pieces
    //      in tetrahedron, edge, side order)
    d.cvol.assign(N, 0.0);
    d.cskew.assign(3 * N, 0.0);
#pragma omp parallel for schedule(dynamic, 1024)
    for (int64_t v = 0; v < N; ++v) {
        double vol = 0.0;
        for (int64_t i = d.nbr_ptr[v]; i < d.nbr_ptr[v + 1]; ++i) vol += d.area[i] * d.dist[i] / 6.0;
        d.cvol[v] = vol;
        double cx = 0.0, cy = 0.0, cz = 0.0;
        for (int64_t q = vt_ptr[v]; q < vt_ptr[v + 1]; ++q) {
            const int64_t t = vt_idx[q];
            const int32_t* tv = &tet[4 * t];
            for (int e = 0; e < 6; ++e) {
                const int32_t vi = tv[kEdgeEnds[e][0]], vj = tv[kEdgeEnds[e][1]];
                if (vi != v && vj != v) continue;
                const V3 pi = P(vi), pj = P(vj);
                const double dist = len3(sub3(pj, pi));
                const V3 pv = vi == v ? pi : pj;
                double pa[2];
                V3 pcen[2];
                pieces(t, e, pa, pcen);
                for (int side = 0; side < 2; ++side) {
                    const double pvol = pa[side] * dist / 6.0;
                    const V3 c = scale3(pvol * 0.75, sub3(pcen[side], pv));
                    cx += c.x;
                    cy += c.y;
                    cz += c.z;
                }
            }
        }
        const double s = 1.0 / vol;
        d.cskew[v] = s * cx;
        d.cskew[N + v] = s * cy;
        d.cskew[2 * N + v] = s * cz;
    }
    pc_area.reset();
    pc_cent.reset();
    ctc.reset();

    std::string e = boundary_subfaces(mesh, bface, d);
    if (!e.empty()) return e;

    // ---- least-squares gradient weights (geom_tet.rs:261-293)
    d.gw.assign(3 * D, 0.0);
    int64_t bad = -1;
#pragma omp parallel for schedule(static)
    for (int64_t v = 0; v < N; ++v) {
        const V3 pc = P(v);
        double m[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        for (int64_t i = d.nbr_ptr[v]; i < d.nbr_ptr[v + 1]; ++i) {
            const V3 dd = sub3(P(d.nbr_idx[i]), pc);
            const double dv[3] = {dd.x, dd.y, dd.z};
            const double omega = 1.0 / (dv[0] * dv[0] + dv[1] * dv[1] + dv[2] * dv[2]);
            for (int r = 0; r < 3; ++r)
                for (int s = 0; s < 3; ++s) m[r][s] += omega * dv[r] * dv[s];
        }
        const double adj[3][3] = {
            {m[1][1] * m[2][2] - m[1][2] * m[2][1], m[0][2] * m[2][1] - m[0][1] * m[2][2], m[0][1] * m[1][2] - m[0][2] * m[1][1]},
            {m[1][2] * m[2][0] - m[1][0] * m[2][2], m[0][0] * m[2][2] - m[0][2] * m[2][0], m[0][2] * m[1][0] - m[0][0] * m[1][2]},
            {m[1][0] * m[2][1] - m[1][1] * m[2][0], m[0][1] * m[2][0] - m[0][0] * m[2][1], m[0][0] * m[1][1] - m[0][1] * m[1][0]},
        };
        const double det = m[0][0] * adj[0][0] + m[0][1] * adj[1][0] + m[0][2] * adj[2][0];
        const double tr = m[0][0] + m[1][1] + m[2][2];
        if (!(det > 1e-12 * tr * tr * tr)) {
#pragma omp critical
            bad = v;
            continue;
        }
        for (int64_t i = d.nbr_ptr[v]; i < d.nbr_ptr[v + 1]; ++i) {
            const V3 dd = sub3(P(d.nbr_idx[i]), pc);
            const double omega = 1.0 / dot3(dd, dd);
            for (int r = 0; r < 3; ++r) d.gw[r * D + i] = omega * (adj[r][0] * dd.x + adj[r][1] * dd.y + adj[r][2] * dd.z) / det;
        }
    }
    if (bad >= 0) return "dual: singular least-squares gradient at vid " + std::to_string(bad);
    return "";
}

}  // namespace vfv
