// Host check of the leading-face geometry of the sweep kernels: for every
// direction and many positions in several box shapes, the brick words and
// masks (table form: face_words + face_table_entry; closed form: face_alu)
// cover exactly the nine sites two steps ahead along the move axis and
// -1..+1 along the two transverse axes, with periodic wrap.  This restates
// checkFront (UpdaterGPUScBFM_AB_Type.cu:420-869) as a set of sites.
#include <cstdio>
#include <cstdlib>
#include <map>
#include "bfm_device.cuh"
using namespace bfm;
int main()
{
    unsigned long long table[192 * 4];
    for (int e = 0; e < 192; ++e) face_table_entry(e, table + e * 4);
    long bad = 0, n = 0;
    const int boxes[4][3] = {{8, 8, 8}, {32, 16, 64}, {256, 256, 256}, {1024, 8, 16}};
    for (auto &L : boxes) {
        Geometry g;
        g.m[0] = dilate3(L[0] - 1);
        g.m[1] = dilate3(L[1] - 1) << 1;
        g.m[2] = dilate3(L[2] - 1) << 2;
        srand(7);
        for (int it = 0; it < 60000; ++it) {
            uint32_t x = rand() % L[0], y = rand() % L[1], z = rand() % L[2];
            if (it < 4096) { x = it % L[0]; y = (it / 7) % L[1]; z = (it / 3) % L[2]; }
            const uint32_t r0 = zcode(x, y, z);
            for (int dir = 0; dir < 6; ++dir) {
                const int ax = dir >> 1, sg = (dir & 1) ? 1 : -1;
                const int bx = ax == 0 ? 1 : 0, cx = ax == 2 ? 1 : 2;
                std::map<uint32_t, unsigned long long> want, tab, alu;
                for (int ib = -1; ib <= 1; ++ib)
                    for (int ic = -1; ic <= 1; ++ic) {
                        int c[3] = {(int)x, (int)y, (int)z};
                        c[ax] += 2 * sg;
                        c[bx] += ib;
                        c[cx] += ic;
                        for (int k = 0; k < 3; ++k) c[k] = ((c[k] % L[k]) + L[k]) % L[k];
                        const uint32_t site = zcode(c[0], c[1], c[2]);
                        want[site >> 6] |= 1ull << (site & 63);
                    }
                const FaceW fw = face_words(r0, dir, g);
                for (int q = 0; q < 4; ++q)
                    if (table[fw.t * 4 + q]) tab[fw.w[q]] |= table[fw.t * 4 + q];
                const FaceM fm = face_alu(r0, dir, g);
                for (int q = 0; q < 4; ++q)
                    if (face_mask(fm, q)) alu[fm.w[q]] |= face_mask(fm, q);
                const uint32_t r1 = zstep(r0, dir, g);
                const uint32_t r1w = (dir & 1) ? zinc(r0, fw.ma, fw.ua) : zdec(r0, fw.ma, fw.ua);
                /* the spill rule of the kernels' lookups (words 1..3 are read when
                 * the transverse start bits lb, lc are >= 2) names exactly the words
                 * the table uses */
                const bool sb = ((fw.t >> 2) & 3u) >= 2u, sc = (fw.t & 3u) >= 2u;
                const bool same = (sb == (table[fw.t * 4 + 1] != 0)) && (sc == (table[fw.t * 4 + 2] != 0)) &&
                                  ((sb && sc) == (table[fw.t * 4 + 3] != 0));
                if (tab != want || alu != want || r1 != r1w || !same) {
                    if (bad < 5) printf("mismatch L=%dx%dx%d x=%u y=%u z=%u dir=%d\n", L[0], L[1], L[2], x, y, z, dir);
                    ++bad;
                }
                ++n;
            }
        }
    }
    printf("checked %ld faces, %ld mismatches\n", n, bad);
    return bad != 0;
}
