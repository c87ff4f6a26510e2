/*
 * bfm_device.cuh -- device arithmetic of the colored BFM sweep.
 *
 * Positions are stored as Z-order (Morton) codes of the wrapped lattice
 * coordinates: bit 3k holds bit k of x, bit 3k+1 bit k of y, bit 3k+2 bit k
 * of z.  This is exactly the lattice index of the reference
 * (linearizeBoxVectorIndex with USE_ZCURVE_FOR_LATTICE,
 * UpdaterGPUScBFM_AB_Type.cu:289-316), so a position is also its own lattice
 * address and its own spatial sort key (.cu:1809-1817).  Unit moves,
 * periodic wrap, the 3x3 leading face and the bond vector are computed
 * directly on the codes with dilated-integer arithmetic:
 *     a (+) unit_k = ((a | ~M_k) + unit_k) & M_k
 *     a (-) b      = (a - b) & M_k
 * where M_k masks the payload bits of axis k inside the box.
 */
#pragma once
#include <cstdint>

namespace bfm {

/* Per-system geometry: payload masks of the three axes, limited to the box
 * (power-of-two edge lengths, so masking is the periodic wrap). */
struct Geometry {
    uint32_t m[3];      /* m[0] = dilated(Lx-1), m[1] = dilated(Ly-1) << 1, m[2] = dilated(Lz-1) << 2 */
    uint32_t open = 0;  /* bit a set: axis a is not periodic */
    uint32_t top[3] = {0, 0, 0}; /* open axis a: dilated(L_a - 2) << a, the highest corner coordinate */
};

__host__ __device__ inline uint32_t dilate3(uint32_t x)
{
    x &= 0x3FFu;
    x = (x | (x << 16)) & 0x030000FFu;
    x = (x | (x << 8)) & 0x0300F00Fu;
    x = (x | (x << 4)) & 0x030C30C3u;
    x = (x | (x << 2)) & 0x09249249u;
    return x;
}

__host__ __device__ inline uint32_t undilate3(uint32_t x)
{
    x &= 0x09249249u;
    x = (x | (x >> 2)) & 0x030C30C3u;
    x = (x | (x >> 4)) & 0x0300F00Fu;
    x = (x | (x >> 8)) & 0x030000FFu;
    x = (x | (x >> 16)) & 0x000003FFu;
    return x;
}

__host__ __device__ inline uint32_t zcode(uint32_t x, uint32_t y, uint32_t z)
{
    return dilate3(x) | (dilate3(y) << 1) | (dilate3(z) << 2);
}

/* the payload mask of axis ax, selected without indexing (an indexed
 * parameter array would live in local memory) */
__host__ __device__ inline uint32_t axis_mask(const Geometry &g, int ax)
{
    return ax == 0 ? g.m[0] : (ax == 1 ? g.m[1] : g.m[2]);
}

/* A move that would take the corner out of the box along a non-periodic
 * axis.  The reference's check (UpdaterGPUScBFM_AB_Type.cu:988-996) lets the
 * corner of a 2x2x2 cube take the coordinates 0 .. L-2 along such an axis
 * (for its unsigned coordinate types; it compares y and z with the x size,
 * which is the same test for cubic boxes).  Positions are kept inside that
 * range from set-up on, so a step is refused exactly when it starts on the
 * edge it is heading for. */
__host__ __device__ inline bool leaves_box(uint32_t r0, int dir, const Geometry &g)
{
    const int ax = dir >> 1;
    if (!((g.open >> ax) & 1u)) return false;
    const uint32_t c = r0 & axis_mask(g, ax);
    const uint32_t top = ax == 0 ? g.top[0] : (ax == 1 ? g.top[1] : g.top[2]);
    return (dir & 1) ? c == top : c == 0u;
}

/* +1 / -1 along one axis with periodic wrap (mask = that axis' payload) */
__host__ __device__ inline uint32_t zinc(uint32_t a, uint32_t mask, uint32_t unit)
{
    return (a & ~mask) | (((a | ~mask) + unit) & mask);
}
__host__ __device__ inline uint32_t zdec(uint32_t a, uint32_t mask, uint32_t unit)
{
    return (a & ~mask) | (((a & mask) - unit) & mask);
}

/* Move direction table of the reference (.cu:1539-1541): 0:-x 1:+x 2:-y 3:+y 4:-z 5:+z */
__host__ __device__ inline uint32_t zstep(uint32_t a, int dir, const Geometry &g)
{
    const int ax = dir >> 1;
    const uint32_t unit = 1u << ax;
    const uint32_t m = axis_mask(g, ax);
    return (dir & 1) ? zinc(a, m, unit) : zdec(a, m, unit);
}

/* Interleaved 9-bit code of the bond vector (b - a) mod 8 per axis.  The
 * bond table is stored in this order (see host table builder). */
__host__ __device__ inline uint32_t zbond(uint32_t b, uint32_t a)
{
    const uint32_t dx = ((b & 0x049u) - (a & 0x049u)) & 0x049u;
    const uint32_t dy = ((b & 0x092u) - (a & 0x092u)) & 0x092u;
    const uint32_t dz = ((b & 0x124u) - (a & 0x124u)) & 0x124u;
    return dx | dy | dz;
}

/* The nine lattice sites of the leading face of a monomer at r0 moving in
 * dir: along the move axis at r0 + 2*D, along the two other axes -1, 0, +1
 * (checkFront, .cu:420-869).  Written out as the 3 values of each transverse
 * axis plus the common part. */
struct Face {
    uint32_t base;      /* all bits except the two transverse axes */
    uint32_t b[3];      /* transverse axis B: coordinate -1, 0, +1 */
    uint32_t c[3];      /* transverse axis C: coordinate -1, 0, +1 */
};

__host__ __device__ inline Face zface(uint32_t r0, int dir, const Geometry &g)
{
    const int ax = dir >> 1;
    const int bx = (ax == 0) ? 1 : 0;
    const int cx = (ax == 2) ? 1 : 2;
    const uint32_t unit = 1u << ax;
    const uint32_t ma = axis_mask(g, ax);
    uint32_t p = (dir & 1) ? zinc(zinc(r0, ma, unit), ma, unit) : zdec(zdec(r0, ma, unit), ma, unit);
    const uint32_t mb = axis_mask(g, bx), mc = axis_mask(g, cx);
    const uint32_t ub = 1u << bx, uc = 1u << cx;
    Face f;
    f.base = p & ~(mb | mc);
    const uint32_t vb = p & mb, vc = p & mc;
    f.b[0] = (vb - ub) & mb;
    f.b[1] = vb;
    f.b[2] = ((vb | ~mb) + ub) & mb;
    f.c[0] = (vc - uc) & mc;
    f.c[1] = vc;
    f.c[2] = ((vc | ~mc) + uc) & mc;
    return f;
}


/* Leading face with its masks in closed form (no table lookups).  The sites
 * of a 4x4x4 brick whose coordinate along axis k lies in a value set V
 * (bit v of V = value v) form a "cylinder" mask; coordinate bits of axis k
 * are bits k and k + 3 of the brick index, so each axis has a closed form:
 *   x: period 16, value v at byte (v >> 1), pattern 0x55 << (v & 1)
 *   y: period 32, value v at half (v >> 1), pattern 0x3333 << 2 (v & 1)
 *   z: value v at word half (v >> 1), pattern 0x0F0F0F0F << 4 (v & 1)
 * written as one multiplication of the spread value set. */
__host__ __device__ __forceinline__ uint32_t cyl_x(uint32_t V)
{
    return ((V & 3u) | ((V & 12u) << 6)) * 0x00550055u;
}
__host__ __device__ __forceinline__ uint32_t cyl_y(uint32_t V)
{
    return ((V & 1u) | ((V & 2u) << 1) | ((V & 4u) << 14) | ((V & 8u) << 15)) * 0x3333u;
}
__host__ __device__ __forceinline__ void cyl_z(uint32_t V, uint32_t &lo, uint32_t &hi)
{
    lo = ((V & 1u) | ((V & 2u) << 3)) * 0x0F0F0F0Fu;
    hi = (((V >> 2) & 1u) | (((V >> 3) & 1u) << 4)) * 0x0F0F0F0Fu;
}

struct FaceM {
    uint32_t w[4];             /* brick words: (b-half, c-half) = (0,0), (1,0), (0,1), (1,1) */
    uint32_t lo[4], hi[4];     /* site masks inside each word (zero: word not touched) */
    uint32_t ma, ua;           /* payload mask and unit of the move axis */
};

/* The face of a move of the monomer at r0 in direction dir: the 3x3 sites
 * two steps ahead along the move axis a, -1..+1 along the transverse axes
 * b, c (b = y for a = x, else x; c = y for a = z, else z). */
__host__ __device__ __forceinline__ FaceM face_alu(uint32_t r0, int dir, const Geometry &g)
{
    const uint32_t ax = (uint32_t)dir >> 1;
    const uint32_t bx = ax == 0u ? 1u : 0u, cx = ax == 2u ? 1u : 2u;
    const uint32_t ma = axis_mask(g, (int)ax), mb = axis_mask(g, (int)bx), mc = axis_mask(g, (int)cx);
    const uint32_t ua = 1u << ax, ub = 1u << bx, uc = 1u << cx;
    const uint32_t two = ua << 3; /* dilated 2 along the move axis */
    const uint32_t pa = (dir & 1) ? (((r0 | ~ma) + two) & ma) : (((r0 & ma) - two) & ma);
    const uint32_t b0 = ((r0 & mb) - ub) & mb;
    const uint32_t b2 = ((r0 | ~mb) + ub) & mb;
    const uint32_t c0 = ((r0 & mc) - uc) & mc;
    const uint32_t c2 = ((r0 | ~mc) + uc) & mc;
    const uint32_t la = ((pa >> ax) & 1u) | ((pa >> (ax + 2u)) & 2u);
    const uint32_t lb = ((b0 >> bx) & 1u) | ((b0 >> (bx + 2u)) & 2u);
    const uint32_t lc = ((c0 >> cx) & 1u) | ((c0 >> (cx + 2u)) & 2u);
    const uint32_t ha = pa >> 6, hb0 = b0 >> 6, hb2 = b2 >> 6, hc0 = c0 >> 6, hc2 = c2 >> 6;
    FaceM f;
    f.w[0] = ha | hb0 | hc0;
    f.w[1] = ha | hb2 | hc0;
    f.w[2] = ha | hb0 | hc2;
    f.w[3] = ha | hb2 | hc2;
    /* value sets: the plane value along a, the transverse ranges split at
     * the brick edge into the near (0) and far (1) brick */
    const uint32_t P = 1u << la;
    const uint32_t tb = 7u << lb, tc = 7u << lc;
    const uint32_t B0 = tb & 15u, B1 = tb >> 4, C0 = tc & 15u, C1 = tc >> 4;
    const uint32_t X0 = cyl_x(ax == 0u ? P : B0), X1 = cyl_x(ax == 0u ? P : B1);
    const uint32_t Y0 = cyl_y(ax == 1u ? P : (ax == 0u ? B0 : C0));
    const uint32_t Y1 = cyl_y(ax == 1u ? P : (ax == 0u ? B1 : C1));
    uint32_t Z0l, Z0h, Z1l, Z1h;
    cyl_z(ax == 2u ? P : C0, Z0l, Z0h);
    cyl_z(ax == 2u ? P : C1, Z1l, Z1h);
    /* word (gb, gc): x takes half gb, z half gc, y half gb when it is the b
     * axis (a = x) and gc otherwise; the plane axis has equal halves */
    const uint32_t t0 = X0 & Y0;
    const uint32_t t1 = X1 & (ax == 0u ? Y1 : Y0);
    const uint32_t t2 = X0 & (ax == 0u ? Y0 : Y1);
    const uint32_t t3 = X1 & Y1;
    f.lo[0] = t0 & Z0l;
    f.hi[0] = t0 & Z0h;
    f.lo[1] = t1 & Z0l;
    f.hi[1] = t1 & Z0h;
    f.lo[2] = t2 & Z1l;
    f.hi[2] = t2 & Z1h;
    f.lo[3] = t3 & Z1l;
    f.hi[3] = t3 & Z1h;
    f.ma = ma;
    f.ua = ua;
    return f;
}

/* Entry e = ((ax * 4 + la) * 4 + lb) * 4 + lc of the face-mask table: for a
 * move along axis ax whose leading face lies in the plane with low
 * coordinate bits la, and whose transverse ranges start at low bits lb, lc,
 * the masks of the nine face sites in the (up to) four bricks it touches,
 * m[gb | gc << 1] (gb, gc: the range spills into the next brick along b, c). */
__host__ __device__ inline void face_table_entry(int e, unsigned long long *m)
{
    const int a = e >> 6, la = (e >> 4) & 3, lb = (e >> 2) & 3, lc = e & 3;
    const int bx = (a == 0) ? 1 : 0;
    const int cx = (a == 2) ? 1 : 2;
    const uint32_t abit = (((uint32_t)la & 1u) | (((uint32_t)la & 2u) << 2)) << a;
    unsigned long long m0 = 0, m1 = 0, m2 = 0, m3 = 0;
    for (int ib = 0; ib < 3; ++ib)
        for (int ic = 0; ic < 3; ++ic) {
            const int vb = lb + ib, vc = lc + ic;
            const int g = (vb >= 4 ? 1 : 0) | (vc >= 4 ? 2 : 0);
            const uint32_t ub = (uint32_t)(vb & 3), uc = (uint32_t)(vc & 3);
            const uint32_t bit = abit | (((ub & 1u) | ((ub & 2u) << 2)) << bx) | (((uc & 1u) | ((uc & 2u) << 2)) << cx);
            const unsigned long long v = 1ull << bit;
            if (g == 0) m0 |= v;
            else if (g == 1) m1 |= v;
            else if (g == 2) m2 |= v;
            else m3 |= v;
        }
    m[0] = m0;
    m[1] = m1;
    m[2] = m2;
    m[3] = m3;
}

/* The four brick words of the face and the index of its masks in the face
 * table ((ax * 4 + la) * 4 + lb) * 4 + lc (la, lb, lc: the low coordinate
 * bits of the plane and of the first transverse values), with the
 * direction constants computed in registers. */
struct FaceW {
    uint32_t w[4];
    uint32_t t;
    uint32_t ma, ua;
};

__host__ __device__ __forceinline__ FaceW face_words(uint32_t r0, int dir, const Geometry &g)
{
    const uint32_t ax = (uint32_t)dir >> 1;
    const uint32_t bx = ax == 0u ? 1u : 0u, cx = ax == 2u ? 1u : 2u;
    const uint32_t ma = axis_mask(g, (int)ax), mb = axis_mask(g, (int)bx), mc = axis_mask(g, (int)cx);
    const uint32_t ua = 1u << ax, ub = 1u << bx, uc = 1u << cx;
    const uint32_t two = ua << 3;
    const uint32_t pa = (dir & 1) ? (((r0 | ~ma) + two) & ma) : (((r0 & ma) - two) & ma);
    const uint32_t b0 = ((r0 & mb) - ub) & mb;
    const uint32_t b2 = ((r0 | ~mb) + ub) & mb;
    const uint32_t c0 = ((r0 & mc) - uc) & mc;
    const uint32_t c2 = ((r0 | ~mc) + uc) & mc;
    const uint32_t la = ((pa >> ax) & 1u) | ((pa >> (ax + 2u)) & 2u);
    const uint32_t lb = ((b0 >> bx) & 1u) | ((b0 >> (bx + 2u)) & 2u);
    const uint32_t lc = ((c0 >> cx) & 1u) | ((c0 >> (cx + 2u)) & 2u);
    const uint32_t ha = pa >> 6, hb0 = b0 >> 6, hb2 = b2 >> 6, hc0 = c0 >> 6, hc2 = c2 >> 6;
    FaceW f;
    f.w[0] = ha | hb0 | hc0;
    f.w[1] = ha | hb2 | hc0;
    f.w[2] = ha | hb0 | hc2;
    f.w[3] = ha | hb2 | hc2;
    f.t = ((ax * 4u + la) * 4u + lb) * 4u + lc;
    f.ma = ma;
    f.ua = ua;
    return f;
}


__host__ __device__ __forceinline__ unsigned long long face_mask(const FaceM &f, int g)
{
    return ((unsigned long long)f.hi[g] << 32) | f.lo[g];
}

/* ------------------------------------------------------------------ RNGs */

enum RngKind { RNG_INTHASH = 1, RNG_SARU = 2, RNG_PHILOX = 3 };

/* Saru generator (S. Worley, HOOMD-blue; rngs/Saru.h:153-170 and
 * :240-261 of the reference): churn (seed, iteration, subsequence) into an
 * LCG + Weyl state and take one output.  The three keys are 32-bit, as in
 * the reference where they are truncated at Saru::init. */
__host__ __device__ inline uint32_t saru(uint32_t k1, uint32_t k2, uint32_t k3)
{
    k3 ^= (k1 << 7) ^ (k2 >> 6);
    k2 += (k1 >> 4) ^ (k3 >> 15);
    k1 ^= (k2 << 9) + (k3 << 8);
    k3 ^= 0xA5366B4Du * ((k2 >> 11) ^ (k1 << 1));
    k2 += 0x72BE1579u * ((k1 << 4) ^ (k3 >> 16));
    k1 ^= 0x3F38A6EDu * ((k3 >> 5) ^ (uint32_t)((int32_t)k2 >> 22));
    k2 += k1 * k3;
    k1 += k3 ^ (k2 >> 2);
    k2 ^= (uint32_t)((int32_t)k2 >> 17);
    uint32_t x = 0x79DEDEA3u * (k1 ^ (uint32_t)((int32_t)k1 >> 14));
    uint32_t y = (x + k2) ^ (uint32_t)((int32_t)x >> 8);
    x = x + y * (y ^ 0xDDDF97F5u);
    y = 0xABCB96F7u + (y >> 1);
    x = 0x4BEB5D59u * x + 0x2600E1F7u;
    y = y + 0x8009D14Bu + ((uint32_t)((int32_t)y >> 31) & 0xDA879ADDu);
    const uint32_t v = (x ^ (x >> 26)) + y;
    return (v ^ (v >> 20)) * 0x6957F5A7u;
}

/* Robert Jenkins' 32-bit integer mix, the reference's IntHash generator
 * (rngs/Hash.h:24-46, :65-69): hash(hash(subsequence) ^ seed). */
__host__ __device__ inline uint32_t jhash(uint32_t a)
{
    a = (a + 0x7ED55D16u) + (a << 12);
    a = (a ^ 0xC761C23Cu) ^ (a >> 19);
    a = (a + 0x165667B1u) + (a << 5);
    a = (a + 0xD3A2646Cu) ^ (a << 9);
    a = (a + 0xFD7046C5u) + (a << 3);
    a = (a ^ 0xB55A4F09u) ^ (a >> 16);
    return a;
}

/* 32x32 -> 64-bit product, high half */
__host__ __device__ inline uint32_t mulhi32(uint32_t a, uint32_t b)
{
#ifdef __CUDA_ARCH__
    return __umulhi(a, b);
#else
    return (uint32_t)(((uint64_t)a * b) >> 32);
#endif
}

/* Philox4x32-10 (Salmon, Moraes, Dror & Shaw, SC'11): ten rounds of two
 * 32x32 multiplications with the Weyl key schedule.  Output word
 * (offset & 3) of the block at counter (offset / 4) + subsequence * 2^64 and
 * key = seed, the stream position of a generator set up with
 * curand_init(seed, subsequence, offset), as rngs/lemonade_philox.h:48-56 of
 * the reference does (checked against curand's own outputs). */
__host__ __device__ inline uint32_t philox_word(uint64_t seed, uint64_t subsequence, uint64_t offset)
{
    const uint64_t blk = offset >> 2;
    uint32_t c0 = (uint32_t)blk, c1 = (uint32_t)(blk >> 32), c2 = (uint32_t)subsequence, c3 = (uint32_t)(subsequence >> 32);
    uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint32_t lo0 = 0xD2511F53u * c0, hi0 = mulhi32(0xD2511F53u, c0);
        const uint32_t lo1 = 0xCD9E8D57u * c2, hi1 = mulhi32(0xCD9E8D57u, c2);
        const uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
        c0 = n0;
        c1 = lo1;
        c2 = n2;
        c3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    const uint32_t w = (uint32_t)(offset & 3u);
    return w == 0 ? c0 : (w == 1 ? c1 : (w == 2 ? c2 : c3));
}

template <int RNG>
__host__ __device__ inline uint32_t draw(uint32_t seed, uint32_t iteration, uint32_t local, uint32_t iterationHi = 0)
{
    if (RNG == RNG_INTHASH) return jhash(jhash(local) ^ seed);
    if (RNG == RNG_PHILOX) return philox_word(seed, local, ((uint64_t)iterationHi << 32) | iteration);
    return saru(seed, iteration, local);
}

/* Direction from the random number: rn % 6 (.cu:967) */
__host__ __device__ inline int direction(uint32_t rn) { return (int)(rn % 6u); }

} // namespace bfm
