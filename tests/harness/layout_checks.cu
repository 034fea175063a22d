// Host-side checks of the index algebra the register-FFT kernels rely on, compiled
// from the kernels' own headers (no GPU needed):
//  * regs_for_blocks: the register caps that give 1..4 resident blocks;
//  * khat_index: the parity-split kernel column is a permutation of 0..ny, and the
//    column pass's read index for bin ky = 2 kk + parity (direct or mirrored) is the
//    entry the builder wrote for that ky;
//  * stage_slot / stage_index: the swizzled staging slots are a permutation inside
//    every group of eight pieces, shifting a piece by a multiple of 32 shifts its slot
//    by the same amount (the per-thread affine addressing of the inverse transform),
//    and a warp's reads of one row spread over the minimum number of wavefronts.
// Prints "ok" and exits 0, or prints the first failure and exits 1.
#include <cstdio>
#include <set>
#include <vector>

#include "fast_kernels.cuh"

using namespace llg;

static int fails = 0;
#define CHECK(c, ...)                      \
    do {                                   \
        if (!(c)) {                        \
            std::printf("FAIL: " __VA_ARGS__); \
            std::printf("\n");             \
            if (++fails > 5) return 1;     \
        }                                  \
    } while (0)

// shared-memory wavefronts of one warp-wide access: 32 banks of 4 bytes, each wavefront
// serves one 4-byte word per bank
static int wavefronts(const std::vector<long>& byte_addr, int bytes) {
    std::vector<std::set<long>> words(32);
    for (long a : byte_addr)
        for (int b = 0; b < bytes; b += 4) words[((a + b) / 4) % 32].insert((a + b) / 4);
    size_t w = 0;
    for (auto& s : words) w = s.size() > w ? s.size() : w;
    return (int)w;
}

template <typename R>
static int check_staging(int L, int G) {
    constexpr int T = 2, PER = 16 / (int)sizeof(cx<R>);
    const int K1 = L + 1, pieces = 3 * K1 * T / PER, groups = (pieces + 7) / 8;
    // permutation inside each group of eight
    for (int gidx = 0; gidx < groups; ++gidx) {
        std::set<int> got;
        for (int q = 0; q < 8; ++q) {
            const int s = stage_slot<R, T>(gidx * 8 + q);
            CHECK(s / 8 == gidx, "stage_slot leaves its group (L %d, piece %d)", L, gidx * 8 + q);
            got.insert(s);
        }
        CHECK((int)got.size() == 8, "stage_slot is not a permutation in group %d (L %d)", gidx, L);
    }
    // affine in multiples of 32 pieces
    for (int p = 0; p < pieces; ++p)
        for (int m = 1; p + 32 * m < pieces + 32; ++m)
            CHECK((stage_slot<R, T>(p + 32 * m) == stage_slot<R, T>(p) + 32 * m), "not affine at piece %d + 32*%d", p, m);
    // a warp of the inverse transform: lane t reads bin k = 2 (t + G r) + par of one row;
    // at most 4 wavefronts (without the swizzle: 8 in FP32, 16 in FP64)
    for (int par = 0; par < 2; ++par)
        for (int half = 0; half < G / 32; ++half)
            for (int r = 0; r < 32 && 2 * (G * r) <= L; ++r) {
                std::vector<long> addr;
                for (int lane = 0; lane < 32; ++lane) {
                    const int t = half * 32 + lane, k = 2 * (t + G * r) + par;
                    if (k > L) continue;
                    addr.push_back((long)stage_index<R, T>(k * T + 0) * (long)sizeof(cx<R>));
                }
                if (addr.empty()) continue;
                const int w = wavefronts(addr, (int)sizeof(cx<R>));
                CHECK(w <= 4, "staged read of L %d, r %d, parity %d takes %d wavefronts", L, r, par, w);
            }
    return 0;
}

int main() {
    // register caps: the sub-partition holding the most warps sets the bound
    CHECK(regs_for_blocks(192, 1) == 255, "192 x 1");
    CHECK(regs_for_blocks(192, 2) == 168, "192 x 2");
    CHECK(regs_for_blocks(192, 3) == 96, "192 x 3");
    CHECK(regs_for_blocks(384, 2) == 80, "384 x 2");
    CHECK(regs_for_blocks(256, 4) == 64, "256 x 4");
    for (int threads : {128, 192, 256, 384})
        for (int b = 1; b <= 4; ++b) {
            const int r = regs_for_blocks(threads, b), warps = b * threads / 32, per = (warps + 3) / 4;
            CHECK(r % 8 == 0 || r == 255, "cap %d not a multiple of 8", r);
            CHECK(per * 32 * r <= 16384, "cap %d over a sub-partition for %d x %d", r, threads, b);
        }
    // parity-split kernel columns
    for (int ny : {16, 32, 128, 1024, 2048}) {
        std::set<int> got;
        for (int ky = 0; ky <= ny; ++ky) got.insert(khat_index(ky, ny));
        CHECK((int)got.size() == ny + 1 && *got.begin() == 0 && *got.rbegin() == ny, "khat_index ny %d", ny);
        const int L = ny;
        for (int par = 0; par < 2; ++par)
            for (int kk = 0; kk < L; ++kk) {
                const int ky = 2 * kk + par;
                const bool up = ky > ny;
                const int read = par ? (up ? ny / 2 + L - kk : ny / 2 + 1 + kk) : (up ? L - kk : kk);
                CHECK(read == khat_index(up ? 2 * L - ky : ky, ny), "column read index ny %d kk %d par %d", ny, kk,
                      par);
            }
    }
    // staging slots of the two-row blocks
    if (check_staging<float>(1024, 32) || check_staging<float>(2048, 64) || check_staging<double>(512, 32) ||
        check_staging<double>(1024, 64))
        return 1;
    if (fails) return 1;
    std::printf("ok\n");
    return 0;
}
