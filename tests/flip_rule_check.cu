// Checks the device flip rules (pt_kernel.cuh: flip_h0, flip_gen) against the
// acceptance rule they implement, bit for bit: a flip of centre spin s with U
// unsatisfied bonds is accepted iff U >= ucut_s or r < thr[s][U].  Every
// combination of (s, sa, ca, sb, cb) sits in one bit of the words; draws and
// thresholds cover the edges (0, equal to a threshold, 0xFFFFFFFF).
// Built and run by tests/test_flip_rule.py; prints the number of mismatches.
#include <cstdio>
#include <cstdint>
#include <vector>

#include "pt_kernel.cuh"

struct Case {
    uint32_t r;
    uint32_t thr[2][7];
    int ucut[2];
};

__global__ void check_kernel(const Case* cases, int n, unsigned* bad) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const Case cs = cases[i];
    // bit b: s0 = b>>4, sa = b&1, ca = (b>>1)&1, sb = (b>>2)&1, cb = (b>>3)&1
    uint32_t s0 = 0, sa = 0, ca = 0, sb = 0, cb = 0;
    for (int b = 0; b < 32; ++b) {
        sa |= ((b >> 0) & 1u) << b;
        ca |= ((b >> 1) & 1u) << b;
        sb |= ((b >> 2) & 1u) << b;
        cb |= ((b >> 3) & 1u) << b;
        s0 |= ((b >> 4) & 1u) << b;
    }
    const uint4 ta = make_uint4(cs.thr[0][0], cs.thr[0][1], cs.thr[0][2], cs.thr[1][0]);
    const uint4 tb = make_uint4(cs.thr[1][1], cs.thr[1][2], cs.thr[1][3], cs.thr[1][4]);
    const uint32_t fl = csg::flip_gen(s0, sa, ca, sb, cb, cs.r, ta, tb, cs.ucut[0], cs.ucut[1]);
    uint32_t want = 0;
    for (int b = 0; b < 32; ++b) {
        const int s = (b >> 4) & 1;
        const int U = (b & 1) + ((b >> 2) & 1) + 2 * (((b >> 1) & 1) + ((b >> 3) & 1));
        const bool acc = U >= cs.ucut[s] || cs.r < cs.thr[s][U];
        want |= (acc ? 1u : 0u) << b;
    }
    if (fl != want) atomicAdd(bad, 1u);
    // the H = 0 rule on the tables where it applies (ucut = 3, equal thresholds)
    if (cs.ucut[0] == 3 && cs.ucut[1] == 3) {
        bool same = true;
        for (int U = 0; U < 3; ++U) same = same && cs.thr[0][U] == cs.thr[1][U];
        if (same) {
            const uint32_t f0 = csg::flip_h0(sa, ca, sb, cb, cs.r, cs.thr[0][0], cs.thr[0][1], cs.thr[0][2]);
            if (f0 != want) atomicAdd(bad + 1, 1u);
        }
    }
}

int main() {
    std::vector<Case> cases;
    uint64_t z = 0x9E3779B97F4A7C15ull;
    auto rnd = [&]() {
        z += 0x9E3779B97F4A7C15ull;
        uint64_t x = z;
        x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
        x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
        return (uint32_t)(x ^ (x >> 31));
    };
    for (int k = 0; k < 20000; ++k) {
        Case c{};
        // cuts as the tables give them: ucut_0 <= 3, ucut_1 <= 5 (0 <= H <= 4)
        c.ucut[0] = (int)(rnd() % 4);
        c.ucut[1] = c.ucut[0] + (int)(rnd() % (6 - c.ucut[0]));
        if (k % 7 == 0) c.ucut[0] = c.ucut[1] = 3;
        for (int s = 0; s < 2; ++s) {
            uint32_t prev = (k % 5 == 0) ? 0u : rnd() >> (rnd() % 32);
            for (int U = 0; U < 7; ++U) {
                if (U >= c.ucut[s]) {
                    c.thr[s][U] = 0xFFFFFFFFu;
                } else {
                    const uint32_t step = rnd() >> (8 + rnd() % 24);
                    prev = prev + step < prev ? 0xFFFFFFFEu : prev + step;  // non-decreasing
                    c.thr[s][U] = prev;
                }
            }
        }
        if (k % 7 == 0)
            for (int U = 0; U < 3; ++U) c.thr[1][U] = c.thr[0][U];
        switch (k % 6) {
            case 0: c.r = 0xFFFFFFFFu; break;
            case 1: c.r = 0u; break;
            case 2: c.r = c.thr[rnd() & 1][rnd() % 5]; break;
            case 3: c.r = c.thr[rnd() & 1][rnd() % 5] - 1u; break;
            default: c.r = rnd(); break;
        }
        cases.push_back(c);
    }
    Case* d = nullptr;
    unsigned* bad = nullptr;
    if (cudaMalloc(&d, cases.size() * sizeof(Case)) != cudaSuccess) return 2;
    if (cudaMalloc(&bad, 2 * sizeof(unsigned)) != cudaSuccess) return 2;
    cudaMemset(bad, 0, 2 * sizeof(unsigned));
    cudaMemcpy(d, cases.data(), cases.size() * sizeof(Case), cudaMemcpyHostToDevice);
    const int n = (int)cases.size();
    check_kernel<<<(n + 127) / 128, 128>>>(d, n, bad);
    unsigned h[2] = {0, 0};
    if (cudaMemcpy(h, bad, sizeof(h), cudaMemcpyDeviceToHost) != cudaSuccess) return 3;
    std::printf("cases %d general-field mismatches %u zero-field mismatches %u\n", n, h[0], h[1]);
    cudaFree(d);
    cudaFree(bad);
    return 0;
}
