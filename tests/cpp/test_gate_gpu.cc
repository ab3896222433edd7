// C++ drop-in check of the gate API shim (include/cufhe_gpu.hpp), written the
// way the reference's test/test_gate_gpu.cc drives cuFHEpp: Ctxt<P> arrays,
// one Stream per "SM slot", every gate in copying form, Synchronize, decrypt.
// Keys come from the client library (TFHEpp's role).  Exit code 0 = all pass.
#include <cstdio>
#include <cstring>
#include <random>
#include <vector>

#include "cufhe_gpu.hpp"
#include "tfhe_client.h"

using namespace cufhe;

static const double kAlpha0 = 9.25e-5, kAlpha1 = 2.98023223876953125e-08;

template <class P>
static int run(const char* name, int gate, int nstreams, int per_stream, const std::vector<int32_t>& key,
               uint64_t seed)
{
    const int n = nstreams * per_stream;
    std::vector<Ctxt<P>> ct(4 * n);
    std::vector<uint8_t> pt(4 * n);
    std::mt19937 rng(seed);
    for (int i = 0; i < 4 * n; i++) {
        pt[i] = rng() & 1;
        tfhe_tlwe32_encrypt(seed, i, key.data(), P::n, pt[i] ? P::mu : 0u - P::mu,
                            P::level == CUFHE_LVL1 ? kAlpha1 : kAlpha0, ct[i].tlwehost.data());
    }
    std::vector<Stream> st(nstreams);
    for (auto& s : st) s.Create();
    for (int i = 0; i < n; i++) {
        Stream s = st[i % nstreams];
        switch (gate) {
        case CUFHE_NAND: Nand<P>(ct[i], ct[i + n], ct[i + 2 * n], s); break;
        case CUFHE_AND: And<P>(ct[i], ct[i + n], ct[i + 2 * n], s); break;
        case CUFHE_OR: Or<P>(ct[i], ct[i + n], ct[i + 2 * n], s); break;
        case CUFHE_XOR: Xor<P>(ct[i], ct[i + n], ct[i + 2 * n], s); break;
        case CUFHE_XNOR: Xnor<P>(ct[i], ct[i + n], ct[i + 2 * n], s); break;
        case CUFHE_NOR: Nor<P>(ct[i], ct[i + n], ct[i + 2 * n], s); break;
        case CUFHE_ANDYN: AndYN<P>(ct[i], ct[i + n], ct[i + 2 * n], s); break;
        case CUFHE_ANDNY: AndNY<P>(ct[i], ct[i + n], ct[i + 2 * n], s); break;
        case CUFHE_ORYN: OrYN<P>(ct[i], ct[i + n], ct[i + 2 * n], s); break;
        case CUFHE_ORNY: OrNY<P>(ct[i], ct[i + n], ct[i + 2 * n], s); break;
        case CUFHE_MUX: Mux<P>(ct[i], ct[i + n], ct[i + 2 * n], ct[i + 3 * n], s); break;
        case CUFHE_NMUX: NMux<P>(ct[i], ct[i + n], ct[i + 2 * n], ct[i + 3 * n], s); break;
        case CUFHE_NOT: Not<P>(ct[i], ct[i + n], s); break;
        case CUFHE_COPY: Copy<P>(ct[i], ct[i + n], s); break;
        }
    }
    Synchronize();
    for (auto& s : st) {
        if (!StreamQuery(s)) return 1;
        s.Destroy();
    }
    int fails = 0;
    for (int i = 0; i < n; i++) {
        const int a = pt[i + n], b = pt[i + 2 * n], c = pt[i + 3 * n];
        int want = 0;
        switch (gate) {
        case CUFHE_NAND: want = !(a & b); break;
        case CUFHE_AND: want = a & b; break;
        case CUFHE_OR: want = a | b; break;
        case CUFHE_XOR: want = a ^ b; break;
        case CUFHE_XNOR: want = !(a ^ b); break;
        case CUFHE_NOR: want = !(a | b); break;
        case CUFHE_ANDYN: want = a & !b; break;
        case CUFHE_ANDNY: want = !a & b; break;
        case CUFHE_ORYN: want = a | !b; break;
        case CUFHE_ORNY: want = !a | b; break;
        case CUFHE_MUX: want = a ? b : c; break;
        case CUFHE_NMUX: want = !(a ? b : c); break;
        case CUFHE_NOT: want = !a; break;
        case CUFHE_COPY: want = a; break;
        }
        uint8_t got = 0;
        tfhe_tlwe32_decrypt_bits(key.data(), P::n, ct[i].tlwehost.data(), 1, &got);
        fails += got != want;
    }
    std::printf("%-6s level %d: %s (%d/%d failures)\n", name, P::level, fails ? "FAIL" : "PASS",
                fails, n);
    return fails ? 1 : 0;
}

// the *_lvl02 gates of the reference's test/test_gate_gpu_lvl02.cc (Ctxt<lvl0>
// I/O through lvl0 -> lvl2 bootstrapping); Not/Copy stay the lvl0 ones
static int run02(const char* name, int gate, int nstreams, int per_stream,
                 const std::vector<int32_t>& key, uint64_t seed)
{
    const int n = nstreams * per_stream;
    std::vector<Ctxt<lvl0param>> ct(4 * n);
    std::vector<uint8_t> pt(4 * n);
    std::mt19937 rng(seed);
    for (int i = 0; i < 4 * n; i++) {
        pt[i] = rng() & 1;
        tfhe_tlwe32_encrypt(seed, i, key.data(), 636, pt[i] ? (1u << 29) : 0u - (1u << 29),
                            kAlpha0, ct[i].tlwehost.data());
    }
    std::vector<Stream> st(nstreams);
    for (auto& s : st) s.Create();
    for (int i = 0; i < n; i++) {
        Stream s = st[i % nstreams];
        Ctxt<lvl0param>&o = ct[i], &a = ct[i + n], &b = ct[i + 2 * n], &c = ct[i + 3 * n];
        switch (gate) {
        case CUFHE_NAND: Nand_lvl02(o, a, b, s); break;
        case CUFHE_OR: Or_lvl02(o, a, b, s); break;
        case CUFHE_ORYN: OrYN_lvl02(o, a, b, s); break;
        case CUFHE_ORNY: OrNY_lvl02(o, a, b, s); break;
        case CUFHE_AND: And_lvl02(o, a, b, s); break;
        case CUFHE_ANDYN: AndYN_lvl02(o, a, b, s); break;
        case CUFHE_ANDNY: AndNY_lvl02(o, a, b, s); break;
        case CUFHE_NOR: Nor_lvl02(o, a, b, s); break;
        case CUFHE_XOR: Xor_lvl02(o, a, b, s); break;
        case CUFHE_XNOR: Xnor_lvl02(o, a, b, s); break;
        case CUFHE_MUX: Mux_lvl02(o, a, b, c, s); break;
        case CUFHE_NMUX: NMux_lvl02(o, a, b, c, s); break;
        case CUFHE_NOT: Not<lvl0param>(o, a, s); break;
        case CUFHE_COPY: Copy<lvl0param>(o, a, s); break;
        }
    }
    Synchronize();
    for (auto& s : st) s.Destroy();
    int fails = 0;
    for (int i = 0; i < n; i++) {
        const int a = pt[i + n], b = pt[i + 2 * n], c = pt[i + 3 * n];
        int want = 0;
        switch (gate) {
        case CUFHE_NAND: want = !(a & b); break;
        case CUFHE_AND: want = a & b; break;
        case CUFHE_OR: want = a | b; break;
        case CUFHE_XOR: want = a ^ b; break;
        case CUFHE_XNOR: want = !(a ^ b); break;
        case CUFHE_NOR: want = !(a | b); break;
        case CUFHE_ANDYN: want = a & !b; break;
        case CUFHE_ANDNY: want = !a & b; break;
        case CUFHE_ORYN: want = a | !b; break;
        case CUFHE_ORNY: want = !a | b; break;
        case CUFHE_MUX: want = a ? b : c; break;
        case CUFHE_NMUX: want = !(a ? b : c); break;
        case CUFHE_NOT: want = !a; break;
        case CUFHE_COPY: want = a; break;
        }
        uint8_t got = 0;
        tfhe_tlwe32_decrypt_bits(key.data(), 636, ct[i].tlwehost.data(), 1, &got);
        fails += got != want;
    }
    std::printf("%-6s lvl02: %s (%d/%d failures)\n", name, fails ? "FAIL" : "PASS", fails, n);
    return fails ? 1 : 0;
}

int main()
{
    const uint64_t seed = 4242;
    std::vector<int32_t> k0(636), k1(1024);
    tfhe_keygen_binary(seed, 0, 636, k0.data());
    tfhe_keygen_binary(seed, 1, 1024, k1.data());
    EvalKey ek;
    ek.keybundle = true;
    ek.bk.resize((size_t)318 * 3 * 8192);
    ek.ksk.resize((size_t)1024 * 7 * 2 * 637);
    tfhe_bk32_gen(seed + 1, k0.data(), 636, k1.data(), 1024, 2, 8, kAlpha1, 1, ek.bk.data());
    tfhe_ksk32_gen(seed + 2, k1.data(), 1024, k0.data(), 636, 2, 7, kAlpha0, ek.ksk.data());
    SetGPUNum(1);
    Initialize(ek);
    const char* names[] = {"Nand", "Or", "OrYN", "OrNY", "And", "AndYN", "AndNY",
                           "Nor",  "Xor", "Xnor", "Not", "Copy", "Mux", "NMux"};
    int bad = 0;
    for (int g = 0; g < 14; g++) {
        bad += run<lvl1param>(names[g], g, 8, 4, k1, seed + 10 + g);
        bad += run<lvl0param>(names[g], g, 8, 4, k0, seed + 30 + g);
    }
    CleanUp();

    std::vector<int32_t> k2(2048);
    tfhe_keygen_binary(seed, 2, 2048, k2.data());
    EvalKey02 ek2;
    ek2.keybundle = true;
    ek2.bk.resize((size_t)318 * 3 * 32768);
    ek2.ksk.resize((size_t)2048 * 7 * 2 * 637);
    tfhe_bk64_gen(seed + 3, k0.data(), 636, k2.data(), 2048, 4, 10, 0x1p-44, 1, ek2.bk.data());
    tfhe_ksk32_gen(seed + 4, k2.data(), 2048, k0.data(), 636, 2, 7, kAlpha0, ek2.ksk.data());
    Initialize_lvl02(ek2, k2);
    for (int g = 0; g < 14; g++) bad += run02(names[g], g, 4, 4, k0, seed + 50 + g);
    CleanUp_lvl02();
    std::printf(bad ? "SOME TESTS FAILED\n" : "ALL TESTS PASSED\n");
    return bad ? 1 : 0;
}
