// Bulk ligand input: the engine's JSON ligand schema parsed natively, and the rigid
// fragments and intra pair lists of every ligand built in one call over host threads.
//
// The document is the one the reference's pybind pipeline serialises with json.dumps and
// hands to rapidjson (api/python/pipeline.cpp:125-139): an object whose members are
// ligands, {"atoms": [[x, y, z, vina_type, ff_type, charge, [1-2/1-3 idx], [1-4 idx]
// (, [[bx, by, bz, V, r2], ...])], ...], "torsions": [[[a, b, c, d], value_deg,
// [[lo_deg, hi_deg], ...], [rotated idx], [gaff2 ...]], ...], "root_atoms": [...]}, with
// the reserved keys "receptor" and "score" skipped (src/format/rapidjson_parser.cpp:54-225).
// The semantics restated per ligand:
//   * 1-2/1-3 pairs: ordered pairs of every atom's list, self pairs dropped (:88-96);
//   * 1-4 pairs: ordered, self pairs and pairs already among the 1-2/1-3 pairs at that
//     point of the atom loop dropped (:98-111);
//   * fragments: torsions with an axis atom in the root set each give a fragment (their
//     rotated atoms and the axis) and add the axis to the root fragment; every other
//     torsion splits the first fragment holding both axis atoms into (fragment n rotated)
//     and (fragment - rotated), both with the axis (split_torsions_into_frags, :227-296);
//   * scored intra pairs: every i < j that is neither a 1-2/1-3 nor a 1-4 pair nor inside
//     one fragment, listed for both atoms in ascending order (:201-221);
//   * angles: float(value) * (3.1415927f / 180) in single precision; torsion ranges only
//     with use_tor_lib, a range crossing +-180 split in two (:150-173), [-pi, pi]
//     otherwise or when no range is valid.
// One thread scans the top-level members while the others build the ligands it has
// found; the export scatters every ligand into the caller's packed arrays.

#include <algorithm>
#include <atomic>
#include <memory>
#include <charconv>
#include <cstdint>
#include <cstring>
#include <limits>
#include <set>
#include <stdexcept>
#include <string>
#include <thread>
#include <utility>
#include <vector>
#if defined(__SSE2__)
#include <emmintrin.h>
#endif

#include "../../include/udock_b200.h"

namespace {

constexpr float PI_F = 3.1415927f;
const float DEG2RAD = PI_F / 180.0f;

struct ParseError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

// ------------------------------------------------------------------ JSON reader
struct Reader {
    const char* p;
    const char* end;

    void ws() {
        while (p < end && (*p == ' ' || *p == '\n' || *p == '\r' || *p == '\t')) p++;
    }
    [[noreturn]] void fail(const char* what) const { throw ParseError(std::string("ligand JSON: ") + what); }
    char peek() {
        ws();
        if (p >= end) fail("unexpected end of input");
        return *p;
    }
    void expect(char c) {
        if (peek() != c) fail((std::string("expected '") + c + "'").c_str());
        p++;
    }
    bool accept(char c) {
        if (peek() == c) {
            p++;
            return true;
        }
        return false;
    }
    static void put_utf8(std::string& s, uint32_t cp) {
        if (cp < 0x80) {
            s += (char)cp;
        } else if (cp < 0x800) {
            s += (char)(0xC0 | (cp >> 6));
            s += (char)(0x80 | (cp & 0x3F));
        } else if (cp < 0x10000) {
            s += (char)(0xE0 | (cp >> 12));
            s += (char)(0x80 | ((cp >> 6) & 0x3F));
            s += (char)(0x80 | (cp & 0x3F));
        } else {
            s += (char)(0xF0 | (cp >> 18));
            s += (char)(0x80 | ((cp >> 12) & 0x3F));
            s += (char)(0x80 | ((cp >> 6) & 0x3F));
            s += (char)(0x80 | (cp & 0x3F));
        }
    }
    uint32_t hex4() {
        if (end - p < 4) fail("bad \\u escape");
        uint32_t v = 0;
        for (int i = 0; i < 4; i++) {
            const char c = *p++;
            v <<= 4;
            if (c >= '0' && c <= '9') v |= (uint32_t)(c - '0');
            else if (c >= 'a' && c <= 'f') v |= (uint32_t)(c - 'a' + 10);
            else if (c >= 'A' && c <= 'F') v |= (uint32_t)(c - 'A' + 10);
            else fail("bad \\u escape");
        }
        return v;
    }
    std::string str() {
        expect('"');
        std::string s;
        while (true) {
            if (p >= end) fail("unterminated string");
            const char c = *p++;
            if (c == '"') break;
            if (c != '\\') {
                s += c;
                continue;
            }
            if (p >= end) fail("unterminated string");
            const char e = *p++;
            switch (e) {
                case '"': s += '"'; break;
                case '\\': s += '\\'; break;
                case '/': s += '/'; break;
                case 'b': s += '\b'; break;
                case 'f': s += '\f'; break;
                case 'n': s += '\n'; break;
                case 'r': s += '\r'; break;
                case 't': s += '\t'; break;
                case 'u': {
                    uint32_t cp = hex4();
                    if (cp >= 0xD800 && cp < 0xDC00 && end - p >= 6 && p[0] == '\\' && p[1] == 'u') {
                        p += 2;
                        const uint32_t lo = hex4();
                        cp = 0x10000 + ((cp - 0xD800) << 10) + (lo - 0xDC00);
                    }
                    put_utf8(s, cp);
                    break;
                }
                default: fail("bad escape");
            }
        }
        return s;
    }
    double num() {
        ws();
        double v = 0.0;
        const char* q = p;
        if (q < end && *q == '+') fail("bad number");
        const auto r = std::from_chars(q, end, v);
        if (r.ec != std::errc()) {
            // the JSON writers of Python emit these for non-finite floats
            if (end - p >= 3 && !strncmp(p, "NaN", 3)) { p += 3; return std::numeric_limits<double>::quiet_NaN(); }
            if (end - p >= 8 && !strncmp(p, "Infinity", 8)) { p += 8; return std::numeric_limits<double>::infinity(); }
            if (end - p >= 9 && !strncmp(p, "-Infinity", 9)) { p += 9; return -std::numeric_limits<double>::infinity(); }
            fail("expected a number");
        }
        p = r.ptr;
        return v;
    }
    int inum() {
        ws();
        // plain integers (the common case) without the floating-point parser
        const char* q = p;
        bool neg = false;
        if (q < end && *q == '-') { neg = true; q++; }
        long long v0 = 0;
        const char* d0 = q;
        while (q < end && *q >= '0' && *q <= '9' && q - d0 < 10) v0 = v0 * 10 + (*q++ - '0');
        if (q > d0 && (q >= end || (*q != '.' && *q != 'e' && *q != 'E' && (*q < '0' || *q > '9')))) {
            p = q;
            v0 = neg ? -v0 : v0;
            if (v0 < -2147483648LL || v0 > 2147483647LL) fail("expected an integer");
            return (int)v0;
        }
        const double v = num();
        if (!(v >= -2147483648.0 && v <= 2147483647.0) || v != (double)(int)v) fail("expected an integer");
        return (int)v;
    }
    // skip one value of any kind (a table-driven scan: only quotes, escapes and brackets
    // matter inside a container)
    void skip() {
        static const struct Cls {
            uint8_t t[256];
            Cls() : t{} {
                t[(uint8_t)'"'] = 1;
                t[(uint8_t)'['] = t[(uint8_t)'{'] = 2;
                t[(uint8_t)']'] = t[(uint8_t)'}'] = 3;
            }
        } cls;
        const char c = peek();
        if (c == '"') {
            p++;
            while (p < end && *p != '"') p += (*p == '\\') ? 2 : 1;
            if (p >= end) fail("unterminated string");
            p++;
        } else if (c == '{' || c == '[') {
            int depth = 0;
            while (p < end) {
#if defined(__SSE2__)
                // 16 bytes at a time up to the next quote or bracket
                const __m128i cq = _mm_set1_epi8('"'), c1 = _mm_set1_epi8('['), c2 = _mm_set1_epi8(']');
                const __m128i c3 = _mm_set1_epi8('{'), c4 = _mm_set1_epi8('}');
                while (end - p >= 16) {
                    const __m128i v = _mm_loadu_si128(reinterpret_cast<const __m128i*>(p));
                    const __m128i m = _mm_or_si128(_mm_or_si128(_mm_cmpeq_epi8(v, cq), _mm_cmpeq_epi8(v, c1)),
                                                   _mm_or_si128(_mm_or_si128(_mm_cmpeq_epi8(v, c2), _mm_cmpeq_epi8(v, c3)),
                                                                _mm_cmpeq_epi8(v, c4)));
                    const int bits = _mm_movemask_epi8(m);
                    if (bits) {
                        p += __builtin_ctz(bits);
                        break;
                    }
                    p += 16;
                }
#endif
                while (p < end && !cls.t[(uint8_t)*p]) p++;
                if (p >= end) break;
                const uint8_t k = cls.t[(uint8_t)*p];
                if (k == 1) {
                    p++;
                    while (p < end && *p != '"') p += (*p == '\\') ? 2 : 1;
                    if (p >= end) fail("unterminated string");
                    p++;
                    continue;
                }
                p++;
                if (k == 2) {
                    depth++;
                } else if (--depth == 0) {
                    return;
                }
            }
            fail("unterminated value");
        } else if (c == 't' && end - p >= 4 && !strncmp(p, "true", 4)) {
            p += 4;
        } else if (c == 'f' && end - p >= 5 && !strncmp(p, "false", 5)) {
            p += 5;
        } else if (c == 'n' && end - p >= 4 && !strncmp(p, "null", 4)) {
            p += 4;
        } else {
            num();
        }
    }
    // call f() once per element of an array
    template <class F>
    void array(F&& f) {
        expect('[');
        if (accept(']')) return;
        while (true) {
            f();
            if (accept(']')) return;
            expect(',');
        }
    }
    // call f(key) once per member of an object (f reads the value)
    template <class F>
    void object(F&& f) {
        expect('{');
        if (accept('}')) return;
        while (true) {
            const std::string k = str();
            expect(':');
            f(k);
            if (accept('}')) return;
            expect(',');
        }
    }
};

// ------------------------------------------------------------------ one ligand
struct Lig {
    std::vector<float> xyz, charges;
    std::vector<int> types, ff;
    std::vector<int> axis;                 // 2 per torsion
    std::vector<float> dihe;
    std::vector<int> range_cnt;            // per torsion
    std::vector<float> ranges;             // 2 per range
    std::vector<int> rot_cnt, rot;         // rotated atoms per torsion
    std::vector<int> pair_cnt, pairs;      // per atom, both directions
    std::vector<int> bias_cnt;             // per atom
    std::vector<float> bias;               // 5 per record
    int n1213 = 0, n14 = 0;
};

struct PairSet {                           // ordered pairs of atom indices
    int n;
    std::vector<uint8_t> m;                // in-range pairs, upper triangle by (a, b), a < b
    std::set<std::pair<int, int>> other;   // pairs with an index outside [0, n)
    int count = 0;
    explicit PairSet(int n_) : n(n_), m((size_t)n_ * n_, 0) {}
    bool has(int a, int b) const {
        if (a > b) std::swap(a, b);
        if (a >= 0 && b < n) return m[(size_t)a * n + b] != 0;
        return other.count({a, b}) != 0;
    }
    void add(int a, int b) {
        if (a > b) std::swap(a, b);
        if (a >= 0 && b < n) {
            uint8_t& v = m[(size_t)a * n + b];
            if (!v) { v = 1; count++; }
        } else if (other.insert({a, b}).second) {
            count++;
        }
    }
};

// Fragments as membership bitmaps over atom indices [base, base + size)
// (split_torsions_into_frags, rapidjson_parser.cpp:227-296).
struct Frags {
    int base = 0, size = 0;
    std::vector<std::vector<uint8_t>> f;
    bool in(size_t fi, int a) const { return f[fi][a - base] != 0; }
};
Frags split_frags(int natom, const std::vector<int>& root, const std::vector<int>& axis,
                  const std::vector<int>& rot_cnt, const std::vector<int>& rot) {
    int lo = 0, hi = natom;                  // index range of every atom the sets can hold
    for (int a : root) { lo = std::min(lo, a); hi = std::max(hi, a + 1); }
    for (int a : axis) { lo = std::min(lo, a); hi = std::max(hi, a + 1); }
    for (int a : rot) { lo = std::min(lo, a); hi = std::max(hi, a + 1); }
    Frags F;
    F.base = lo;
    F.size = hi - lo;
    const int T = (int)rot_cnt.size();
    std::vector<uint8_t> rootm(F.size, 0);
    for (int a : root) rootm[a - lo] = 1;
    std::vector<uint8_t> frag0 = rootm;
    std::vector<int> rest;
    std::vector<size_t> roff(T + 1, 0);
    for (int k = 0; k < T; k++) roff[k + 1] = roff[k] + rot_cnt[k];
    for (int k = 0; k < T; k++) {
        const int a0 = axis[2 * k] - lo, a1 = axis[2 * k + 1] - lo;
        if (rootm[a0] || rootm[a1]) {
            frag0[a0] = frag0[a1] = 1;
            std::vector<uint8_t> m(F.size, 0);
            for (size_t q = roff[k]; q < roff[k + 1]; q++) m[rot[q] - lo] = 1;
            m[a0] = m[a1] = 1;
            F.f.push_back(std::move(m));
        } else {
            rest.push_back(k);
        }
    }
    F.f.push_back(std::move(frag0));
    std::vector<uint8_t> tor(F.size, 0);
    for (int k : rest) {
        const int a0 = axis[2 * k] - lo, a1 = axis[2 * k + 1] - lo;
        for (size_t fi = 0; fi < F.f.size(); fi++) {
            if (F.f[fi][a0] && F.f[fi][a1]) {
                for (size_t q = roff[k]; q < roff[k + 1]; q++) tor[rot[q] - lo] = 1;
                std::vector<uint8_t> f2(F.size, 0);
                std::vector<uint8_t>& f1 = F.f[fi];
                for (int a = 0; a < F.size; a++) {
                    if (f1[a] && !tor[a]) { f2[a] = 1; f1[a] = 0; }
                }
                f1[a0] = f1[a1] = 1;
                f2[a0] = f2[a1] = 1;
                for (size_t q = roff[k]; q < roff[k + 1]; q++) tor[rot[q] - lo] = 0;
                F.f.push_back(std::move(f2));
                break;
            }
        }
    }
    return F;
}

void parse_ligand(Reader& r, Lig& L, bool use_tor_lib) {
    std::vector<int> root;
    bool have_atoms = false;
    // the atoms' 1-2/1-3 and 1-4 lists are kept flat until natom is known: entries
    // (atom, partner) in reading order
    static thread_local std::vector<int> l1213, l14;
    l1213.clear();
    l14.clear();
    r.object([&](const std::string& key) {
        if (key == "atoms") {
            have_atoms = true;
            r.array([&]() {
                const int ia = (int)L.types.size();
                int field = 0;
                int nb = 0;
                r.array([&]() {
                    switch (field) {
                        case 0: case 1: case 2: L.xyz.push_back((float)r.num()); break;
                        case 3: L.types.push_back(r.inum()); break;
                        case 4: L.ff.push_back(r.inum()); break;
                        case 5: L.charges.push_back((float)r.num()); break;
                        case 6: r.array([&]() { l1213.push_back(ia); l1213.push_back(r.inum()); }); break;
                        case 7: r.array([&]() { l14.push_back(ia); l14.push_back(r.inum()); }); break;
                        case 8:
                            r.array([&]() {
                                int kk = 0;
                                r.array([&]() {
                                    const float v = (float)r.num();
                                    if (kk < 5) L.bias.push_back(v);
                                    kk++;
                                });
                                if (kk < 5) r.fail("a bias record needs 5 numbers");
                                nb++;
                            });
                            break;
                        default: r.skip();
                    }
                    field++;
                });
                if (field < 8) r.fail("an atom row needs at least 8 fields");
                L.bias_cnt.push_back(nb);
            });
        } else if (key == "torsions") {
            r.array([&]() {
                int field = 0;
                std::vector<int> four;
                std::vector<float> rl;
                std::vector<int> rot;
                float dihe = 0.f;
                r.array([&]() {
                    switch (field) {
                        case 0: r.array([&]() { four.push_back(r.inum()); }); break;
                        case 1: dihe = (float)r.num() * DEG2RAD; break;
                        case 2:
                            r.array([&]() {
                                int kk = 0;
                                float lo = 0.f, hi = 0.f;
                                r.array([&]() {
                                    const float v = (float)r.num() * DEG2RAD;
                                    if (kk == 0) lo = v;
                                    else if (kk == 1) hi = v;
                                    kk++;
                                });
                                if (kk < 2) r.fail("a torsion range needs 2 numbers");
                                if (!use_tor_lib) return;
                                if (lo < hi) {
                                    rl.push_back(lo); rl.push_back(hi);
                                } else if (lo > 0.f && hi < 0.f) {
                                    rl.push_back(lo); rl.push_back(PI_F);
                                    rl.push_back(-PI_F); rl.push_back(hi);
                                }
                            });
                            break;
                        case 3: r.array([&]() { rot.push_back(r.inum()); }); break;
                        default: r.skip();
                    }
                    field++;
                });
                if (field < 4 || four.size() < 4) r.fail("a torsion needs [[a, b, c, d], value, ranges, rotated]");
                if (rl.empty()) { rl.push_back(-PI_F); rl.push_back(PI_F); }
                L.axis.push_back(four[1]);
                L.axis.push_back(four[2]);
                L.dihe.push_back(dihe);
                L.range_cnt.push_back((int)rl.size() / 2);
                L.ranges.insert(L.ranges.end(), rl.begin(), rl.end());
                L.rot_cnt.push_back((int)rot.size());
                L.rot.insert(L.rot.end(), rot.begin(), rot.end());
            });
        } else if (key == "root_atoms") {
            r.array([&]() { root.push_back(r.inum()); });
        } else {
            r.skip();
        }
    });
    if (!have_atoms) r.fail("a ligand needs \"atoms\"");
    const int n = (int)L.types.size();
    // 1-2/1-3 and 1-4 pairs in the atom loop's order (rapidjson_parser.cpp:88-111)
    PairSet p1213(n), p14(n);
    size_t u = 0, v = 0;
    for (int ia = 0; ia < n; ia++) {
        for (; u < l1213.size() && l1213[u] == ia; u += 2)
            if (l1213[u + 1] != ia) p1213.add(ia, l1213[u + 1]);
        for (; v < l14.size() && l14[v] == ia; v += 2)
            if (l14[v + 1] != ia && !p1213.has(ia, l14[v + 1])) p14.add(ia, l14[v + 1]);
    }
    L.n1213 = p1213.count;
    L.n14 = p14.count;
    // fragment membership as bit masks per atom
    const Frags F = split_frags(n, root, L.axis, L.rot_cnt, L.rot);
    const size_t nf = F.f.size();
    const int nw = ((int)nf + 63) / 64;
    std::vector<uint64_t> member((size_t)n * nw, 0);
    for (size_t fi = 0; fi < nf; fi++)
        for (int a = 0; a < n; a++)
            if (F.in(fi, a)) member[(size_t)a * nw + fi / 64] |= 1ull << (fi % 64);
    auto same_frag = [&](int a, int b) {
        for (int w = 0; w < nw; w++)
            if (member[(size_t)a * nw + w] & member[(size_t)b * nw + w]) return true;
        return false;
    };
    // scored pairs, per atom in ascending order (rapidjson_parser.cpp:201-221)
    std::vector<uint8_t> ok((size_t)n * n, 0);
    for (int i = 0; i < n; i++)
        for (int j = i + 1; j < n; j++)
            if (!p1213.m[(size_t)i * n + j] && !p14.m[(size_t)i * n + j] && !same_frag(i, j))
                ok[(size_t)i * n + j] = ok[(size_t)j * n + i] = 1;
    L.pair_cnt.assign(n, 0);
    for (int a = 0; a < n; a++)
        for (int b = 0; b < n; b++)
            if (ok[(size_t)a * n + b]) {
                L.pairs.push_back(b);
                L.pair_cnt[a]++;
            }
}

}  // namespace

struct ud_ligset {
    std::vector<std::string> names;
    std::vector<Lig> ligs;
    struct Base {
        size_t a, t, r, rot, pr, b;
    };
    std::vector<Base> base;              // per-ligand starts in the packed arrays, nlig + 1
};

namespace {
thread_local std::string g_topo_err;

unsigned pick_threads(int nthreads) {
    return nthreads > 0 ? (unsigned)nthreads : std::max(1u, std::thread::hardware_concurrency());
}

// Top-level members found by one thread while the others build the ligands already found:
// spans and ligands live in fixed blocks (never moved), spans published by a release counter.
struct SpanQueue {
    static constexpr size_t BS = 4096;
    struct Item {
        const char* b;
        const char* e;
    };
    std::vector<std::unique_ptr<Item[]>> blocks;
    std::vector<std::unique_ptr<Lig[]>> ligs;
    std::atomic<size_t> published{0};
    std::atomic<bool> done{false};
    explicit SpanQueue(size_t len) : blocks(len / (BS * 6) + 2), ligs(blocks.size()) {}  // a member takes >= 6 bytes
    // called by the scanning thread only; the block is allocated before it is published
    bool push(size_t i, const char* b, const char* e) {
        if (i / BS >= blocks.size()) return false;
        if (i % BS == 0) {
            blocks[i / BS].reset(new Item[BS]);
            ligs[i / BS].reset(new Lig[BS]);
        }
        blocks[i / BS][i % BS] = Item{b, e};
        published.store(i + 1, std::memory_order_release);
        return true;
    }
};
}  // namespace

extern "C" {

const char* ud_ligset_last_error(void) { return g_topo_err.c_str(); }

int ud_ligset_parse_json(const char* json, size_t len, int use_tor_lib, int nthreads, ud_ligset** out) {
    if (!json || !out) {
        g_topo_err = "invalid arguments";
        return UD_EINVAL;
    }
    *out = nullptr;
    ud_ligset* S = new (std::nothrow) ud_ligset();
    if (!S) {
        g_topo_err = "out of host memory";
        return UD_EINVAL;
    }
    try {
        SpanQueue Q(len);
        const unsigned nt = pick_threads(nthreads);
        std::atomic<size_t> claimed{0};
        std::atomic<bool> stop{false};
        std::vector<std::string> errs(nt + 1);
        // workers take members in order as the scan publishes them
        auto work = [&](unsigned w) {
            try {
                while (!stop.load(std::memory_order_relaxed)) {
                    const size_t i = claimed.fetch_add(1);
                    while (i >= Q.published.load(std::memory_order_acquire)) {
                        if (stop.load(std::memory_order_relaxed)) return;
                        if (Q.done.load(std::memory_order_acquire) && i >= Q.published.load(std::memory_order_acquire))
                            return;
                        std::this_thread::yield();
                    }
                    const SpanQueue::Item it = Q.blocks[i / SpanQueue::BS][i % SpanQueue::BS];
                    Reader lr{it.b, it.e};
                    parse_ligand(lr, Q.ligs[i / SpanQueue::BS][i % SpanQueue::BS], use_tor_lib != 0);
                }
            } catch (const std::exception& e) {
                errs[w] = e.what();
                stop.store(true);
            }
        };
        std::vector<std::thread> th;
        for (unsigned w = 1; w < nt; w++) th.emplace_back(work, w);
        // the scan, on this thread (rapidjson_parser.cpp:54-64: the reserved keys are skipped)
        size_t n = 0;
        try {
            Reader r{json, json + len};
            r.object([&](const std::string& key) {
                if (key == "receptor" || key == "score") {
                    r.skip();
                    return;
                }
                r.ws();
                const char* b = r.p;
                r.skip();
                S->names.push_back(key);
                if (!Q.push(n++, b, r.p)) r.fail("more members than the document can hold");
            });
            r.ws();
            if (r.p != r.end) r.fail("trailing characters after the document");
        } catch (const std::exception& e) {
            errs[nt] = e.what();
            stop.store(true);
        }
        Q.done.store(true, std::memory_order_release);
        work(0);                                  // then this thread builds ligands too
        for (auto& t : th) t.join();
        for (const auto& e : errs)
            if (!e.empty()) throw ParseError(e);
        S->ligs.resize(n);
        for (size_t i = 0; i < n; i++) S->ligs[i] = std::move(Q.ligs[i / SpanQueue::BS][i % SpanQueue::BS]);
        S->base.assign(n + 1, ud_ligset::Base{0, 0, 0, 0, 0, 0});
        for (size_t i = 0; i < n; i++) {
            const Lig& L = S->ligs[i];
            const auto& B = S->base[i];
            S->base[i + 1] = ud_ligset::Base{B.a + L.types.size(), B.t + L.dihe.size(), B.r + L.ranges.size() / 2,
                                             B.rot + L.rot.size(), B.pr + L.pairs.size(), B.b + L.bias.size() / 5};
        }
        const auto& tot = S->base[n];
        if (tot.a > 2147483647u || tot.pr > 2147483647u || tot.rot > 2147483647u || tot.t > 2147483647u)
            throw ParseError("ligand JSON: the set exceeds 2^31 atoms, torsions or pair entries; split it");
    } catch (const std::exception& e) {
        g_topo_err = e.what();
        delete S;
        return UD_EINVAL;
    }
    *out = S;
    return UD_OK;
}

int ud_ligset_sizes(const ud_ligset* S, long long* out8) {
    if (!S || !out8) {
        g_topo_err = "invalid arguments";
        return UD_EINVAL;
    }
    size_t nb = 0;
    for (const auto& n : S->names) nb += n.size();
    const auto& t = S->base.back();
    out8[0] = (long long)S->names.size();
    out8[1] = (long long)t.a;
    out8[2] = (long long)t.t;
    out8[3] = (long long)t.r;
    out8[4] = (long long)t.rot;
    out8[5] = (long long)t.pr;
    out8[6] = (long long)t.b;
    out8[7] = (long long)nb;
    return UD_OK;
}

int ud_ligset_export(const ud_ligset* S, int* atom_off, float* xyz, int* types, int* ff_types, float* charges,
                     int* tors_off, int* axis, float* dihedrals, int* range_off, float* ranges, int* rot_off,
                     int* rot_atoms, int* pair_off, int* pairs, int* bias_off, float* bias, int* n_pairs_1213,
                     int* n_pairs_14, long long* name_off, char* names) {
    if (!S) {
        g_topo_err = "invalid arguments";
        return UD_EINVAL;
    }
    const size_t nl = S->ligs.size();
    const auto& tot = S->base[nl];
    auto copy = [](auto* dst, const auto& v) {
        if (dst && !v.empty()) memcpy(dst, v.data(), v.size() * sizeof(v[0]));
    };
    // every ligand scattered to its place, ligands shared among the host threads
    std::atomic<size_t> next{0};
    auto work = [&]() {
        while (true) {
            const size_t b0 = next.fetch_add(64);
            if (b0 >= nl) break;
            for (size_t i = b0; i < std::min(nl, b0 + 64); i++) {
                const Lig& L = S->ligs[i];
                const auto& B = S->base[i];
                if (atom_off) atom_off[i] = (int)B.a;
                if (tors_off) tors_off[i] = (int)B.t;
                copy(xyz ? xyz + 3 * B.a : nullptr, L.xyz);
                copy(charges ? charges + B.a : nullptr, L.charges);
                copy(types ? types + B.a : nullptr, L.types);
                copy(ff_types ? ff_types + B.a : nullptr, L.ff);
                copy(axis ? axis + 2 * B.t : nullptr, L.axis);
                copy(dihedrals ? dihedrals + B.t : nullptr, L.dihe);
                copy(ranges ? ranges + 2 * B.r : nullptr, L.ranges);
                copy(rot_atoms ? rot_atoms + B.rot : nullptr, L.rot);
                copy(pairs ? pairs + B.pr : nullptr, L.pairs);
                copy(bias ? bias + 5 * B.b : nullptr, L.bias);
                size_t r = B.r, q = B.rot;
                for (size_t k = 0; k < L.dihe.size(); k++) {
                    if (range_off) range_off[B.t + k] = (int)r;
                    if (rot_off) rot_off[B.t + k] = (int)q;
                    r += L.range_cnt[k];
                    q += L.rot_cnt[k];
                }
                size_t pr = B.pr, bb = B.b;
                for (size_t a = 0; a < L.types.size(); a++) {
                    if (pair_off) pair_off[B.a + a] = (int)pr;
                    if (bias_off) bias_off[B.a + a] = (int)bb;
                    pr += L.pair_cnt[a];
                    bb += L.bias_cnt[a];
                }
                if (n_pairs_1213) n_pairs_1213[i] = L.n1213;
                if (n_pairs_14) n_pairs_14[i] = L.n14;
            }
        }
    };
    const unsigned nt = (unsigned)std::min<size_t>(pick_threads(0), std::max<size_t>(1, nl / 256));
    std::vector<std::thread> th;
    for (unsigned w = 1; w < nt; w++) th.emplace_back(work);
    work();
    for (auto& t : th) t.join();
    if (atom_off) atom_off[nl] = (int)tot.a;
    if (tors_off) tors_off[nl] = (int)tot.t;
    if (range_off) range_off[tot.t] = (int)tot.r;
    if (rot_off) rot_off[tot.t] = (int)tot.rot;
    if (pair_off) pair_off[tot.a] = (int)tot.pr;
    if (bias_off) bias_off[tot.a] = (int)tot.b;
    if (name_off) {
        long long o = 0;
        for (size_t i = 0; i < nl; i++) {
            name_off[i] = o;
            if (names) memcpy(names + o, S->names[i].data(), S->names[i].size());
            o += (long long)S->names[i].size();
        }
        name_off[nl] = o;
    }
    return UD_OK;
}

void ud_ligset_free(ud_ligset* S) { delete S; }

}  // extern "C"
