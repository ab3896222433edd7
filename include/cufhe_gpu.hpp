// cufhe_gpu.hpp -- the reference's C++ gate API (include/cufhe_gpu.cuh:42-358)
// rebuilt as a header-only layer over the C-ABI of cufhe_b200.h.
//
// Names, argument order and semantics follow the reference: SetGPUNum,
// Initialize(EvalKey), CleanUp, Synchronize, Stream (round-robin device,
// Create/Destroy), StreamQuery, Ctxt<P> (pinned host TLWE + one device
// buffer per GPU, non-copyable), the 14 gates in copying (Nand, ...) and
// device-resident (gNand, ...) forms, for P = lvl0param (blind rotation then
// key switching) and P = lvl1param (key switching then blind rotation), and
// the lvl02 path: Initialize_lvl02 / CleanUp_lvl02 and Nand_lvl02 ...
// NMux_lvl02 on Ctxt<lvl0param> (include/cufhe_gpu.cuh:59-64, :332-358).
// Differences: TFHEpp types are replaced by the plain-array EvalKey below,
// and errors throw cufhe::Error instead of printing and exiting.
#pragma once

#include <array>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "cufhe_b200.h"

namespace cufhe {

struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

inline void check(int rc, const char* what)
{
    if (rc != CUFHE_OK) throw Error(rc, std::string(what) + ": " + cufhe_last_error());
}

// TFHEpp::lvl0param / lvl1param stand-ins (Torus32, mu = 1/8)
struct lvl0param {
    using T = uint32_t;
    static constexpr uint32_t n = 636;
    static constexpr uint32_t k = 1;
    static constexpr int level = CUFHE_LVL0;
    static constexpr uint32_t mu = 1u << 29;
};
struct lvl1param {
    using T = uint32_t;
    static constexpr uint32_t n = 1024;
    static constexpr uint32_t k = 1;
    static constexpr int level = CUFHE_LVL1;
    static constexpr uint32_t mu = 1u << 29;
};

template <class P>
using TLWE = std::array<typename P::T, P::k * P::n + 1>;

// TFHEpp::EvalKey stand-in: bootstrapping key and lvl1->lvl0 key-switching
// key in TFHEpp layouts (see cufhe_keyview)
struct EvalKey {
    std::vector<uint32_t> bk;
    std::vector<uint32_t> ksk;
    bool keybundle = true;
};

// The EvalKey members Initialize_lvl02 reads (getbk<lvl02param>,
// getiksk<lvl20param>): BK<lvl2> in uint64 words, lvl2->lvl0 KSK
struct EvalKey02 {
    std::vector<uint64_t> bk;
    std::vector<uint32_t> ksk;
    bool keybundle = true;
};

inline void SetGPUNum(int n) { check(cufhe_set_gpu_num(n), "SetGPUNum"); }

inline void Initialize(const EvalKey& ek)
{
    cufhe_keyview kv{ek.bk.data(), ek.bk.size(), ek.ksk.data(), ek.ksk.size(),
                     ek.keybundle ? 1 : 0};
    check(cufhe_initialize(&kv), "Initialize");
}

inline void CleanUp() { check(cufhe_cleanup(), "CleanUp"); }

// Initialize_lvl02(ek, sk) -- src/cufhe_gates_gpu.cu:75-90 (the secret key
// argument is unused there too)
inline void Initialize_lvl02(const EvalKey02& ek)
{
    cufhe_keyview02 kv{ek.bk.data(), ek.bk.size(), ek.ksk.data(), ek.ksk.size(),
                       ek.keybundle ? 1 : 0};
    check(cufhe_initialize_lvl02(&kv), "Initialize_lvl02");
}
template <class SecretKey>
inline void Initialize_lvl02(const EvalKey02& ek, const SecretKey&)
{
    Initialize_lvl02(ek);
}
inline void CleanUp_lvl02() { check(cufhe_cleanup_lvl02(), "CleanUp_lvl02"); }
inline void Synchronize() { check(cufhe_synchronize(), "Synchronize"); }

namespace detail {
inline int& stream_count()
{
    static int c = 0;
    return c;
}
}  // namespace detail

// class Stream (include/cufhe_gpu.cuh:162-199): the default constructor picks
// a device round robin; Create() makes the CUDA stream.  A Stream that was
// never created runs on the default stream of the current device.
class Stream {
   public:
    Stream() : st_(nullptr), device_(detail::stream_count()++ % cufhe_get_gpu_num()) {}
    explicit Stream(int device_id) : st_(nullptr), device_(device_id) { detail::stream_count()++; }
    void Create() { check(cufhe_stream_create(&st_, device_), "Stream::Create"); }
    void Destroy()
    {
        check(cufhe_stream_destroy(st_), "Stream::Destroy");
        st_ = nullptr;
    }
    cufhe_stream_t st() const { return st_; }
    int device_id() const { return device_; }

   private:
    cufhe_stream_t st_;
    int device_;
};

inline bool StreamQuery(Stream st)
{
    const int r = cufhe_stream_query(st.st());
    if (r < 0) check(r, "StreamQuery");
    return r == 1;
}

// Ctxt<P> (include/cufhe_gpu.cuh:78-121): pinned host TLWE + device buffers
template <class P>
struct Ctxt {
    Ctxt()
    {
        // page-locking is an optimisation: neighbouring Ctxts share pages and a
        // second registration of a page fails, which (as in the reference,
        // which ignores it) leaves that copy pageable but correct
        (void)cufhe_host_register(tlwehost.data(), sizeof(tlwehost));
        const int g = cufhe_get_gpu_num();
        tlwedevices.resize(g);
        for (int i = 0; i < g; i++) {
            void* p = nullptr;
            check(cufhe_ctxt_alloc(&p, sizeof(tlwehost), i), "Ctxt device alloc");
            tlwedevices[i] = static_cast<typename P::T*>(p);
        }
    }
    ~Ctxt()
    {
        cufhe_host_unregister(tlwehost.data());
        for (size_t i = 0; i < tlwedevices.size(); i++) cufhe_ctxt_free(tlwedevices[i], (int)i);
    }
    Ctxt(const Ctxt&) = delete;
    Ctxt& operator=(const Ctxt&) = delete;

    alignas(64) TLWE<P> tlwehost;
    std::vector<typename P::T*> tlwedevices;
};

namespace detail {
template <class P>
inline void gate_copy(int g, const char* name, Ctxt<P>& out, Ctxt<P>& a, Ctxt<P>* b, Ctxt<P>* c,
                      Stream st)
{
    const int d = st.device_id();
    check(cufhe_gate_copy(g, P::level, out.tlwehost.data(), out.tlwedevices[d], a.tlwehost.data(),
                          a.tlwedevices[d], b ? b->tlwehost.data() : nullptr,
                          b ? b->tlwedevices[d] : nullptr, c ? c->tlwehost.data() : nullptr,
                          c ? c->tlwedevices[d] : nullptr, st.st()),
          name);
}
inline void gate_copy02(int g, const char* name, Ctxt<lvl0param>& out, Ctxt<lvl0param>& a,
                        Ctxt<lvl0param>* b, Ctxt<lvl0param>* c, Stream st)
{
    const int d = st.device_id();
    check(cufhe_gate_copy(g, CUFHE_LVL02, out.tlwehost.data(), out.tlwedevices[d],
                          a.tlwehost.data(), a.tlwedevices[d], b ? b->tlwehost.data() : nullptr,
                          b ? b->tlwedevices[d] : nullptr, c ? c->tlwehost.data() : nullptr,
                          c ? c->tlwedevices[d] : nullptr, st.st()),
          name);
}
template <class P>
inline void gate_dev(int g, const char* name, Ctxt<P>& out, Ctxt<P>& a, Ctxt<P>* b, Ctxt<P>* c,
                     Stream st)
{
    const int d = st.device_id();
    check(cufhe_gate(g, P::level, out.tlwedevices[d], a.tlwedevices[d],
                     b ? b->tlwedevices[d] : nullptr, c ? c->tlwedevices[d] : nullptr, st.st()),
          name);
}
}  // namespace detail

#define CUFHE_BINARY_GATE(Name, ID)                                                    \
    template <class P>                                                                 \
    inline void Name(Ctxt<P>& out, Ctxt<P>& in0, Ctxt<P>& in1, Stream st)              \
    {                                                                                  \
        detail::gate_copy<P>(ID, #Name, out, in0, &in1, nullptr, st);                  \
    }                                                                                  \
    template <class P>                                                                 \
    inline void g##Name(Ctxt<P>& out, Ctxt<P>& in0, Ctxt<P>& in1, Stream st)           \
    {                                                                                  \
        detail::gate_dev<P>(ID, "g" #Name, out, in0, &in1, nullptr, st);               \
    }                                                                                  \
    inline void Name##_lvl02(Ctxt<lvl0param>& out, Ctxt<lvl0param>& in0,               \
                             Ctxt<lvl0param>& in1, Stream st)                          \
    {                                                                                  \
        detail::gate_copy02(ID, #Name "_lvl02", out, in0, &in1, nullptr, st);          \
    }

CUFHE_BINARY_GATE(Nand, CUFHE_NAND)
CUFHE_BINARY_GATE(Or, CUFHE_OR)
CUFHE_BINARY_GATE(OrYN, CUFHE_ORYN)
CUFHE_BINARY_GATE(OrNY, CUFHE_ORNY)
CUFHE_BINARY_GATE(And, CUFHE_AND)
CUFHE_BINARY_GATE(AndYN, CUFHE_ANDYN)
CUFHE_BINARY_GATE(AndNY, CUFHE_ANDNY)
CUFHE_BINARY_GATE(Nor, CUFHE_NOR)
CUFHE_BINARY_GATE(Xor, CUFHE_XOR)
CUFHE_BINARY_GATE(Xnor, CUFHE_XNOR)
#undef CUFHE_BINARY_GATE

// Mux(out, inc, in1, in0) = inc ? in1 : in0 (src/cufhe_gates_gpu.cu:768-824)
template <class P>
inline void Mux(Ctxt<P>& out, Ctxt<P>& inc, Ctxt<P>& in1, Ctxt<P>& in0, Stream st)
{
    detail::gate_copy<P>(CUFHE_MUX, "Mux", out, inc, &in1, &in0, st);
}
template <class P>
inline void gMux(Ctxt<P>& out, Ctxt<P>& inc, Ctxt<P>& in1, Ctxt<P>& in0, Stream st)
{
    detail::gate_dev<P>(CUFHE_MUX, "gMux", out, inc, &in1, &in0, st);
}
template <class P>
inline void NMux(Ctxt<P>& out, Ctxt<P>& inc, Ctxt<P>& in1, Ctxt<P>& in0, Stream st)
{
    detail::gate_copy<P>(CUFHE_NMUX, "NMux", out, inc, &in1, &in0, st);
}
template <class P>
inline void gNMux(Ctxt<P>& out, Ctxt<P>& inc, Ctxt<P>& in1, Ctxt<P>& in0, Stream st)
{
    detail::gate_dev<P>(CUFHE_NMUX, "gNMux", out, inc, &in1, &in0, st);
}
inline void Mux_lvl02(Ctxt<lvl0param>& out, Ctxt<lvl0param>& inc, Ctxt<lvl0param>& in1,
                      Ctxt<lvl0param>& in0, Stream st)
{
    detail::gate_copy02(CUFHE_MUX, "Mux_lvl02", out, inc, &in1, &in0, st);
}
inline void NMux_lvl02(Ctxt<lvl0param>& out, Ctxt<lvl0param>& inc, Ctxt<lvl0param>& in1,
                       Ctxt<lvl0param>& in0, Stream st)
{
    detail::gate_copy02(CUFHE_NMUX, "NMux_lvl02", out, inc, &in1, &in0, st);
}
template <class P>
inline void Not(Ctxt<P>& out, Ctxt<P>& in, Stream st)
{
    detail::gate_copy<P>(CUFHE_NOT, "Not", out, in, nullptr, nullptr, st);
}
template <class P>
inline void gNot(Ctxt<P>& out, Ctxt<P>& in, Stream st)
{
    detail::gate_dev<P>(CUFHE_NOT, "gNot", out, in, nullptr, nullptr, st);
}
template <class P>
inline void Copy(Ctxt<P>& out, Ctxt<P>& in, Stream st)
{
    detail::gate_copy<P>(CUFHE_COPY, "Copy", out, in, nullptr, nullptr, st);
}
template <class P>
inline void gCopy(Ctxt<P>& out, Ctxt<P>& in, Stream st)
{
    detail::gate_dev<P>(CUFHE_COPY, "gCopy", out, in, nullptr, nullptr, st);
}
template <class P>
inline void CopyOnHost(Ctxt<P>& out, Ctxt<P>& in)
{
    out.tlwehost = in.tlwehost;
}

}  // namespace cufhe
