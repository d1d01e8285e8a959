// sv_image.cu -- the path's input format: PNG and Netpbm decoding
// (stereonet.py:244-324 read_pnm, 3204-3628 inflate / zlib_decompress /
// _unfilter / read_png / read_image).
//
// Decoding is sequential by nature (DEFLATE's bit stream, PNG's row
// filters that depend on the left and upper neighbours), so it runs on the
// host into raw samples -- one to two bytes per channel instead of eight --
// and only those cross to the GPU, where one thread per pixel forms the FP64
// rgb and gray values exactly as the reference does (s * 1/(2^depth - 1),
// palette / 255.0, gray = 0.299 r + 0.587 g + 0.114 b left to right).
//
// The inflater follows RFC 1951 (stored, fixed and dynamic Huffman blocks,
// canonical codes decoded a bit at a time); the zlib wrapper checks RFC
// 1950's method, header check and preset-dictionary bit as the reference
// does and, like it, ignores the Adler-32 trailer and the chunk CRCs.

#include <algorithm>
#include <atomic>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "sv_common.cuh"

namespace sv {
namespace {

// ----------------------------------------------------------------- inflate
struct BitIn {
    const uint8_t *p;
    size_t n, pos;
    uint64_t buf = 0;
    int cnt = 0;
    bool fail = false;
    void fill() {
        while (cnt <= 56 && pos < n) {
            buf |= (uint64_t)p[pos++] << cnt;
            cnt += 8;
        }
    }
    uint32_t get(int k) {                 // k <= 32, LSB first
        if (cnt < k) {
            fill();
            if (cnt < k) { fail = true; return 0; }
        }
        const uint32_t v = (uint32_t)(buf & ((1ull << k) - 1));
        buf >>= k;
        cnt -= k;
        return v;
    }
    void align() {
        const int d = cnt & 7;
        buf >>= d;
        cnt -= d;
    }
};

// Canonical Huffman code: counts per length, symbols in code order, and a
// direct table over the next kFast bits (entry = length << 9 | symbol, 0
// for codes longer than kFast or unused).
constexpr int kFast = 10;
struct Code {
    int count[16];
    int sym[320];
    uint16_t fast[1 << kFast];
};

bool build(Code &c, const uint8_t *len, int n) {
    int offs[16], next[16];
    for (int i = 0; i < 16; ++i) c.count[i] = 0;
    for (int s = 0; s < n; ++s) c.count[len[s]]++;
    c.count[0] = 0;
    int left = 1;                                   // over-subscription check
    for (int l = 1; l < 16; ++l) {
        left <<= 1;
        left -= c.count[l];
        if (left < 0) return false;
    }
    offs[1] = 0;
    for (int l = 1; l < 15; ++l) offs[l + 1] = offs[l] + c.count[l];
    for (int s = 0; s < n; ++s)
        if (len[s]) c.sym[offs[len[s]]++] = s;
    // first code of each length (RFC 1951 section 3.2.2)
    int code = 0;
    next[0] = 0;
    for (int l = 1; l < 16; ++l) {
        code = (code + c.count[l - 1]) << 1;
        next[l] = code;
    }
    memset(c.fast, 0, sizeof(c.fast));
    for (int s = 0; s < n; ++s) {
        const int l = len[s];
        if (!l) continue;
        const int cd = next[l]++;
        if (l > kFast) continue;
        int rev = 0;                                // codes arrive MSB first
        for (int k = 0; k < l; ++k) rev |= ((cd >> k) & 1) << (l - 1 - k);
        for (int i = rev; i < (1 << kFast); i += 1 << l) c.fast[i] = (uint16_t)((l << 9) | s);
    }
    return true;
}

// One symbol: the direct table when the code is short, else extend the code
// one bit at a time until it falls inside the range of its length.
int decode(BitIn &b, const Code &c) {
    if (b.cnt < kFast) b.fill();
    const int e = c.fast[b.buf & ((1u << kFast) - 1)];
    if (e && (e >> 9) <= b.cnt) {
        b.buf >>= e >> 9;
        b.cnt -= e >> 9;
        return e & 511;
    }
    int code = 0, first = 0, index = 0;
    for (int l = 1; l < 16; ++l) {
        code |= (int)b.get(1);
        if (b.fail) return -1;
        const int cnt = c.count[l];
        if (code - first < cnt) return c.sym[index + code - first];
        index += cnt;
        first = (first + cnt) << 1;
        code <<= 1;
    }
    return -1;
}

// RFC 1951 section 3.2.5 tables
const int kLenBase[29] = {3, 4, 5, 6, 7, 8, 9, 10, 11, 13, 15, 17, 19, 23, 27,
                          31, 35, 43, 51, 59, 67, 83, 99, 115, 131, 163, 195, 227, 258};
const int kLenExtra[29] = {0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 2, 2, 2,
                           2, 3, 3, 3, 3, 4, 4, 4, 4, 5, 5, 5, 5, 0};
const int kDistBase[30] = {1, 2, 3, 4, 5, 7, 9, 13, 17, 25, 33, 49, 65, 97, 129,
                           193, 257, 385, 513, 769, 1025, 1537, 2049, 3073, 4097,
                           6145, 8193, 12289, 16385, 24577};
const int kDistExtra[30] = {0, 0, 0, 0, 1, 1, 2, 2, 3, 3, 4, 4, 5, 5, 6,
                            6, 7, 7, 8, 8, 9, 9, 10, 10, 11, 11, 12, 12, 13, 13};
const int kClOrder[19] = {16, 17, 18, 0, 8, 7, 9, 6, 10, 5, 11, 4, 12, 3, 13, 2, 14, 1, 15};

// The fixed codes of RFC 1951 section 3.2.6, built once (thread-safe
// static initialisation).
struct FixedCodes {
    Code lit, dist;
    FixedCodes() {
        uint8_t l[288], d[30];
        for (int s = 0; s < 288; ++s) l[s] = s < 144 ? 8 : s < 256 ? 9 : s < 280 ? 7 : 8;
        for (int s = 0; s < 30; ++s) d[s] = 5;
        build(lit, l, 288);
        build(dist, d, 30);
    }
};
const FixedCodes &fixed_codes() {
    static const FixedCodes f;
    return f;
}

// Decoded bytes, growing on demand up to `limit` (a stream that inflates
// past it is rejected rather than exhausting memory).
struct Out {
    std::vector<uint8_t> v;
    size_t size = 0, limit;
    bool room(size_t k) {
        if (size + k > limit) return false;
        if (size + k > v.size()) v.resize(std::max(size + k, std::min(limit, 2 * v.size() + 4096)));
        return true;
    }
};

// The symbols of one Huffman block.  The bit buffer and the output cursor
// live in locals for the loop (stores of output bytes may alias anything
// reachable through a pointer); the slow bit-at-a-time decode and buffer
// growth write them back first.
bool codes(BitIn &b, const Code &lit, const Code &dist, Out &out) {
    uint64_t buf = b.buf;
    int cnt = b.cnt;
    size_t pos = b.pos, size = out.size;
    const uint8_t *const p = b.p;
    const size_t n = b.n;
    uint8_t *o = out.v.data();
    size_t cap = out.v.size();
    bool ok = false;
    auto refill = [&]() {
        if (pos + 8 <= n) {                 // whole-word refill; bytes past cnt are
            uint64_t w;                     // re-read at the same bit position later
            memcpy(&w, p + pos, 8);
            buf |= w << cnt;
            pos += (size_t)((63 - cnt) >> 3);
            cnt |= 56;
        } else {
            while (cnt <= 56 && pos < n) {
                buf |= (uint64_t)p[pos++] << cnt;
                cnt += 8;
            }
        }
    };
    auto sync_out = [&]() { b.buf = buf; b.cnt = cnt; b.pos = pos; };
    auto sync_in = [&]() { buf = b.buf; cnt = b.cnt; pos = b.pos; };
    auto sym = [&](const Code &c) -> int {
        if (cnt < 15) refill();
        const int e = c.fast[buf & ((1u << kFast) - 1)];
        if (e && (e >> 9) <= cnt) {
            buf >>= e >> 9;
            cnt -= e >> 9;
            return e & 511;
        }
        sync_out();
        const int s = decode(b, c);
        sync_in();
        return s;
    };
    auto bits = [&](int k) -> uint32_t {      // k <= 13 after a refill to >= 15
        if (cnt < k) {
            refill();
            if (cnt < k) { cnt = -1; return 0; }
        }
        const uint32_t v = (uint32_t)(buf & ((1u << k) - 1));
        buf >>= k;
        cnt -= k;
        return v;
    };
    for (;;) {
        const int s = sym(lit);
        if (s < 0) break;
        if (size + 258 > cap) {                 // room for the longest match, or
            out.size = size;                    // as much as the limit leaves
            const size_t want = std::min(out.limit, size + 258) - size;
            if (want == 0 || !out.room(want)) break;
            o = out.v.data();
            cap = out.v.size();
        }
        if (s < 256) {
            if (size >= cap) break;
            o[size++] = (uint8_t)s;
        } else if (s == 256) {
            ok = true;
            break;
        } else {
            const int li = s - 257;
            if (li >= 29) break;
            const int len = kLenBase[li] + (int)bits(kLenExtra[li]);
            if (cnt < 0) break;
            const int ds = sym(dist);
            if (ds < 0 || ds >= 30) break;
            const size_t d = (size_t)kDistBase[ds] + bits(kDistExtra[ds]);
            if (cnt < 0 || d > size || size + (size_t)len > cap) break;
            uint8_t *q = o + size;
            for (int k = 0; k < len; ++k) q[k] = q[(ptrdiff_t)k - (ptrdiff_t)d];  // may overlap
            size += (size_t)len;
        }
    }
    if (cnt < 0) return false;
    sync_out();
    out.size = size;
    return ok;
}

bool inflate_raw(const uint8_t *p, size_t n, Out &out) {
    BitIn b{p, n, 0};
    for (;;) {
        const uint32_t last = b.get(1), type = b.get(2);
        if (b.fail) return false;
        if (type == 0) {
            b.align();
            const uint32_t len = b.get(16), nlen = b.get(16);
            if (b.fail || (len ^ 0xffffu) != nlen || !out.room(len)) return false;
            uint32_t k = 0;
            for (; k < len && b.cnt >= 8; ++k) out.v[out.size++] = (uint8_t)b.get(8);
            b.buf &= b.cnt ? ((1ull << b.cnt) - 1) : 0;   // drop read-ahead bytes
            const uint32_t rest = len - k;
            if (b.pos + rest > b.n) return false;
            memcpy(out.v.data() + out.size, b.p + b.pos, rest);
            out.size += rest;
            b.pos += rest;
        } else if (type == 1) {
            if (!codes(b, fixed_codes().lit, fixed_codes().dist, out)) return false;
        } else if (type == 2) {
            const int nlen = (int)b.get(5) + 257, ndist = (int)b.get(5) + 1,
                      ncode = (int)b.get(4) + 4;
            if (b.fail || nlen > 286 || ndist > 30) return false;
            uint8_t cl[19] = {0};
            for (int k = 0; k < ncode; ++k) cl[kClOrder[k]] = (uint8_t)b.get(3);
            Code clc;
            if (b.fail || !build(clc, cl, 19)) return false;
            // a repeat may run past nlen + ndist: the surplus is dropped, as
            // the reference slices the list it built
            uint8_t lens[320 + 138] = {0};
            int k = 0;
            while (k < nlen + ndist) {
                const int s = decode(b, clc);
                if (s < 0) return false;
                if (s < 16) {
                    lens[k++] = (uint8_t)s;
                } else {
                    int rep = 0;
                    uint8_t v = 0;
                    if (s == 16) {
                        if (k == 0) return false;
                        v = lens[k - 1];
                        rep = 3 + (int)b.get(2);
                    } else if (s == 17) {
                        rep = 3 + (int)b.get(3);
                    } else {
                        rep = 11 + (int)b.get(7);
                    }
                    if (b.fail) return false;
                    while (rep--) lens[k++] = v;
                }
            }
            Code lit, dist;
            if (!build(lit, lens, nlen) || !build(dist, lens + nlen, ndist)) return false;
            if (!codes(b, lit, dist, out)) return false;
        } else {
            return false;
        }
        if (last) return true;
    }
}

// PNG's Paeth predictor (stereonet.py:3436-3453), written with the
// distances |b - c|, |a - c| and |a + b - 2c| so it compiles to selects.
inline int paeth(int a, int b, int c) {
    const int pa = abs(b - c), pb = abs(a - c), pc = abs(a + b - 2 * c);
    // selects as masks: a branch here would follow the pixel data
    const int m1 = -(int)(pb <= pc), m2 = -(int)((pa <= pb) & (pa <= pc));
    const int bc = (b & m1) | (c & ~m1);
    return (a & m2) | (bc & ~m2);
}

// The sequential filters (Sub, Average, Paeth) for BPP bytes per pixel:
// the left pixel (a) and the upper-left one (c) ride in registers, so the
// dependency along the row does not go through memory; the filter type and
// whether a row lies above are template arguments, so the per-byte loop
// carries no branch.  i < BPP is done by the caller.
template <int BPP, int FT, bool UP>
void unfilter_seq_t(const uint8_t *__restrict__ row, const uint8_t *__restrict__ up,
                    uint8_t *__restrict__ o, int stride) {
    int a[BPP], c[BPP];
    for (int k = 0; k < BPP; ++k) {
        a[k] = o[k];
        c[k] = UP ? up[k] : 0;
    }
    int i = BPP;
    for (; i + BPP <= stride; i += BPP) {
        for (int k = 0; k < BPP; ++k) {
            const int b = UP ? up[i + k] : 0;
            int v;
            if (FT == 1) v = row[i + k] + a[k];
            else if (FT == 3) v = row[i + k] + ((a[k] + b) >> 1);
            else v = row[i + k] + paeth(a[k], b, c[k]);
            a[k] = v & 0xFF;
            c[k] = b;
            o[i + k] = (uint8_t)v;
        }
    }
    for (int k = 0; i + k < stride; ++k) {      // a partial pixel (sub-byte rows)
        const int b = UP ? up[i + k] : 0;
        const int v = FT == 1 ? row[i + k] + a[k]
                    : FT == 3 ? row[i + k] + ((a[k] + b) >> 1)
                              : row[i + k] + paeth(a[k], b, c[k]);
        o[i + k] = (uint8_t)v;
    }
}

template <int BPP>
void unfilter_seq(int ft, const uint8_t *__restrict__ row, const uint8_t *__restrict__ up,
                  uint8_t *__restrict__ o, int stride) {
    if (ft == 1)
        up ? unfilter_seq_t<BPP, 1, true>(row, up, o, stride)
           : unfilter_seq_t<BPP, 1, false>(row, up, o, stride);
    else if (ft == 3)
        up ? unfilter_seq_t<BPP, 3, true>(row, up, o, stride)
           : unfilter_seq_t<BPP, 3, false>(row, up, o, stride);
    else
        up ? unfilter_seq_t<BPP, 4, true>(row, up, o, stride)
           : unfilter_seq_t<BPP, 4, false>(row, up, o, stride);
}

// One row of _unfilter (stereonet.py:3456-3496); `up` is NULL on row 0,
// where the row above reads as zeros.  The filter type selects the loop.
void unfilter_row(int ft, const uint8_t *__restrict__ row, const uint8_t *__restrict__ up,
                  uint8_t *__restrict__ o, int stride, int bpp) {
    const int head = bpp < stride ? bpp : stride;
    if (ft == 0 || (ft == 2 && !up)) {
        memcpy(o, row, (size_t)stride);
        return;
    }
    if (ft == 2) {
        for (int i = 0; i < stride; ++i) o[i] = (uint8_t)(row[i] + up[i]);
        return;
    }
    // first pixel: a = c = 0, so Sub gives row, Average row + b/2, Paeth row + b
    for (int i = 0; i < head; ++i) {
        const int b = up ? up[i] : 0;
        o[i] = (uint8_t)(row[i] + (ft == 1 ? 0 : ft == 3 ? (b >> 1) : b));
    }
    if (ft == 4 && !up) ft = 1;                     // paeth(a, 0, 0) = a
    switch (bpp) {
    case 1: unfilter_seq<1>(ft, row, up, o, stride); break;
    case 2: unfilter_seq<2>(ft, row, up, o, stride); break;
    case 3: unfilter_seq<3>(ft, row, up, o, stride); break;
    case 4: unfilter_seq<4>(ft, row, up, o, stride); break;
    case 6: unfilter_seq<6>(ft, row, up, o, stride); break;
    default: unfilter_seq<8>(ft, row, up, o, stride); break;
    }
}

uint32_t be32(const uint8_t *p) {
    return ((uint32_t)p[0] << 24) | ((uint32_t)p[1] << 16) | ((uint32_t)p[2] << 8) | p[3];
}

// Walks PNG chunks as read_png does (stereonet.py:3515-3540): a chunk
// cut short by the end of the file keeps the bytes that are there and ends
// the walk; IEND ends it too.
struct Chunks {
    const uint8_t *p;
    size_t n, pos = 8;
    const uint8_t *type = nullptr, *body = nullptr;
    size_t len = 0;
    bool next() {
        if (pos + 8 > n) return false;
        const size_t declared = be32(p + pos);
        type = p + pos + 4;
        body = p + pos + 8;
        len = declared < n - pos - 8 ? declared : n - pos - 8;
        pos += 12 + declared;
        return true;
    }
    bool is(const char *t) const { return memcmp(type, t, 4) == 0; }
};

}  // namespace

// ------------------------------------------------------- GPU conversion
// One thread per pixel: samples -> FP64 rgb and gray (read_png 3556-3598,
// read_pnm 290-322).
__global__ void k_raw_to_float(const uint8_t *__restrict__ raw, sv_raw_image d,
                               double *__restrict__ gray, double *__restrict__ rgb) {
    const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    const long npix = (long)d.width * d.height;
    if (i >= npix) return;
    const int y = (int)(i / d.width), x = (int)(i - (long)y * d.width);
    const uint8_t *row = raw + (long)y * d.stride;
    unsigned s[3] = {0, 0, 0};
    const int ch = d.channels;
    if (d.depth == 8) {
        for (int c = 0; c < (ch < 3 ? ch : 3); ++c) s[c] = row[x * ch + c];
    } else if (d.depth == 16) {
        for (int c = 0; c < (ch < 3 ? ch : 3); ++c)
            s[c] = ((unsigned)row[2 * (x * ch + c)] << 8) | row[2 * (x * ch + c) + 1];
    } else {
        const int bit = x * d.depth;
        const int byte = row[bit >> 3];
        s[0] = (unsigned)(byte >> (8 - d.depth - (bit & 7))) & ((1u << d.depth) - 1u);
    }
    double r, g, b;
    if (d.colortype == 3) {
        const int p = 3 * (int)s[0];
        r = __ddiv_rn((double)d.palette[p], 255.0);
        g = __ddiv_rn((double)d.palette[p + 1], 255.0);
        b = __ddiv_rn((double)d.palette[p + 2], 255.0);
    } else if (d.colortype == 0 || d.colortype == 4) {
        r = g = b = __dmul_rn((double)s[0], d.inv);
    } else {
        r = __dmul_rn((double)s[0], d.inv);
        g = __dmul_rn((double)s[1], d.inv);
        b = __dmul_rn((double)s[2], d.inv);
    }
    if (rgb) {
        rgb[3 * i] = r;
        rgb[3 * i + 1] = g;
        rgb[3 * i + 2] = b;
    }
    if (gray) {
        // read_pnm keeps a one-channel sample as its gray value
        gray[i] = d.colortype == 0 && d.kind == SV_IMAGE_PNM
                      ? r
                      : __dadd_rn(__dadd_rn(__dmul_rn(0.299, r), __dmul_rn(0.587, g)),
                                  __dmul_rn(0.114, b));
    }
}

}  // namespace sv

using namespace sv;

namespace {

int fail(const char *msg) {
    set_error("%s", msg);
    return SV_ERR_PARAM;
}

// Header fields of a PNG (no decompression).
int png_header(const uint8_t *p, size_t n, sv_raw_image *d) {
    static const uint8_t sig[8] = {0x89, 'P', 'N', 'G', '\r', '\n', 0x1a, '\n'};
    if (n < 8 || memcmp(p, sig, 8) != 0) return fail("not a PNG file");
    Chunks ck{p, n};
    bool have = false;
    while (ck.next()) {
        if (ck.is("IHDR")) {
            if (ck.len < 13) return fail("PNG IHDR chunk too short");
            const uint8_t *b = ck.body;
            const uint32_t w = be32(b), h = be32(b + 4);
            if (w < 1 || h < 1 || w > (1u << 27) || h > (1u << 27) || (uint64_t)w * h > (1ull << 31))
                return fail("bad PNG size");
            d->width = (int)w;
            d->height = (int)h;
            d->depth = b[8];
            d->colortype = b[9];
            d->interlace = b[12];
            have = true;
        } else if (ck.is("PLTE")) {
            d->palette_len = (int)(ck.len < 768 ? ck.len : 768);
            memset(d->palette, 0, sizeof(d->palette));
            memcpy(d->palette, ck.body, (size_t)d->palette_len);
        } else if (ck.is("IEND")) {
            break;
        }
    }
    if (!have) return fail("PNG without IHDR");
    if (d->interlace) return fail("Adam7 interlaced PNG is not supported; re-save without interlacing");
    const int dp = d->depth, ct = d->colortype;
    if (dp != 1 && dp != 2 && dp != 4 && dp != 8 && dp != 16) return fail("unsupported PNG bit depth");
    const int chs[7] = {1, 0, 3, 1, 2, 0, 4};
    if (ct < 0 || ct > 6 || !chs[ct]) return fail("unsupported PNG colour type");
    if ((dp < 8 && ct != 0 && ct != 3) || (dp == 16 && ct == 3))
        return fail("PNG bit depth not allowed for its colour type");
    d->kind = SV_IMAGE_PNG;
    d->channels = chs[ct];
    d->stride = (int)(((long)d->width * d->channels * dp + 7) / 8);
    d->inv = dp == 16 ? 1.0 / 65535.0 : 1.0 / ((1 << dp) - 1);
    return SV_OK;
}

void pnm_tokens(const uint8_t *p, size_t n, size_t &i, long tok[3], int &nt) {
    nt = 0;
    while (nt < 3 && i < n) {
        const uint8_t ch = p[i];
        if (ch == '#') {
            while (i < n && p[i] != 10 && p[i] != 13) ++i;
        } else if (ch == ' ' || ch == 9 || ch == 10 || ch == 13) {
            ++i;
        } else {
            long v = 0;
            while (i < n && p[i] != ' ' && p[i] != 9 && p[i] != 10 && p[i] != 13) {
                if (p[i] < '0' || p[i] > '9' || v > (1l << 40)) v = -1;
                if (v >= 0) v = v * 10 + (p[i] - '0');
                ++i;
            }
            tok[nt++] = v;
        }
    }
}

int pnm_header(const uint8_t *p, size_t n, sv_raw_image *d, size_t *payload) {
    if (n < 2 || p[0] != 'P' || (p[1] != '2' && p[1] != '3' && p[1] != '5' && p[1] != '6'))
        return fail("not a PGM/PPM file");
    size_t i = 2;
    long tok[3];
    int nt;
    pnm_tokens(p, n, i, tok, nt);
    if (nt < 3 || tok[0] < 1 || tok[1] < 1 || tok[2] < 1 || tok[2] > 65535 ||
        tok[0] > (1l << 27) || tok[1] > (1l << 27) || tok[0] * tok[1] > (1l << 31))
        return fail("bad PGM/PPM header");
    d->kind = SV_IMAGE_PNM;
    d->width = (int)tok[0];
    d->height = (int)tok[1];
    d->maxval = (int)tok[2];
    d->channels = (p[1] == '3' || p[1] == '6') ? 3 : 1;
    d->colortype = d->channels == 3 ? 2 : 0;
    d->ascii = p[1] == '2' || p[1] == '3';
    // samples are handed to the GPU as 16-bit big-endian when ASCII or
    // maxval > 255, else as the file's bytes
    d->depth = (!d->ascii && d->maxval < 256) ? 8 : 16;
    d->stride = d->width * d->channels * (d->depth / 8);
    d->inv = 1.0 / d->maxval;
    *payload = i;
    return SV_OK;
}

}  // namespace

extern "C" {

int sv_image_info(const uint8_t *data, size_t n, sv_raw_image *desc) {
    if (!data || !desc) { set_error("NULL argument"); return SV_ERR_NULL; }
    memset(desc, 0, sizeof(*desc));
    static const uint8_t sig[8] = {0x89, 'P', 'N', 'G', '\r', '\n', 0x1a, '\n'};
    if (n >= 8 && !memcmp(data, sig, 8)) return png_header(data, n, desc);
    size_t payload;
    return pnm_header(data, n, desc, &payload);
}

int sv_image_decode_raw(const uint8_t *data, size_t n, uint8_t *raw, size_t raw_bytes,
                        sv_raw_image *desc) {
    int rc = sv_image_info(data, n, desc);
    if (rc) return rc;
    const size_t need = (size_t)desc->stride * desc->height;
    if (!raw || raw_bytes < need) {
        set_error("raw buffer needs %zu bytes", need);
        return SV_ERR_WORKSPACE;
    }
    if (desc->kind == SV_IMAGE_PNM) {
        size_t pos;
        sv_raw_image tmp;
        pnm_header(data, n, &tmp, &pos);
        const long count = (long)desc->width * desc->height * desc->channels;
        if (desc->ascii) {
            size_t i = pos;
            for (long k = 0; k < count; ++k) {
                while (i < n && (data[i] == ' ' || (data[i] >= 9 && data[i] <= 13)))
                    ++i;                                // bytes.split() whitespace
                long v = 0;
                bool any = false;
                while (i < n && data[i] >= '0' && data[i] <= '9') {
                    if (v <= 65535) v = v * 10 + (data[i] - '0');
                    ++i;
                    any = true;
                }
                if (!any || v > 65535) return fail("bad PGM/PPM sample");
                raw[2 * k] = (uint8_t)(v >> 8);
                raw[2 * k + 1] = (uint8_t)(v & 255);
            }
        } else {
            pos += 1;                                   // one whitespace byte after maxval
            const size_t bytes = (size_t)count * (desc->maxval < 256 ? 1 : 2);
            if (pos + bytes > n) return fail("truncated PGM/PPM payload");
            memcpy(raw, data + pos, bytes);
        }
        return SV_OK;
    }
    // PNG: concatenate IDAT (the palette was read with the header)
    std::vector<uint8_t> idat;
    Chunks ck{data, n};
    while (ck.next()) {
        if (ck.is("IDAT")) idat.insert(idat.end(), ck.body, ck.body + ck.len);
        else if (ck.is("IEND")) break;
    }
    if (desc->colortype == 3 && desc->palette_len == 0) return fail("indexed PNG with no PLTE chunk");
    // zlib_decompress (stereonet.py:3421-3433)
    if (idat.size() < 2) return fail("zlib stream too short");
    const uint8_t cmf = idat[0], flg = idat[1];
    if ((cmf & 0x0F) != 8) return fail("unsupported zlib compression method");
    if ((((unsigned)cmf << 8) | flg) % 31 != 0) return fail("zlib header checksum failed");
    if (flg & 0x20) return fail("zlib preset dictionary not supported");
    const int stride = desc->stride, H = desc->height;
    const size_t image_bytes = (size_t)(stride + 1) * H;
    Out z;
    z.limit = image_bytes + ((size_t)64 << 20);     // trailing data the reference would ignore
    z.v.resize(image_bytes);
    if (!inflate_raw(idat.data() + 2, idat.size() - 2, z)) return fail("corrupt DEFLATE stream");
    if (z.size < image_bytes) return fail("PNG image data too short");
    // _unfilter (stereonet.py:3456-3496)
    const int bpp = (desc->channels * desc->depth) / 8 > 1 ? (desc->channels * desc->depth) / 8 : 1;
    const uint8_t *src = z.v.data();
    for (int y = 0; y < H; ++y) {
        const int ft = src[0];
        if (ft > 4) {
            set_error("unknown PNG filter type %d on row %d", ft, y);
            return SV_ERR_PARAM;
        }
        unfilter_row(ft, src + 1, y > 0 ? raw + (size_t)(y - 1) * stride : nullptr,
                     raw + (size_t)y * stride, stride, bpp);
        src += stride + 1;
    }
    if (desc->colortype == 3) {               // palette[3 p + 2] must exist
        const int dp = desc->depth;
        for (int y = 0; y < H; ++y)
            for (int x = 0; x < desc->width; ++x) {
                const int bit = x * dp;
                const int p = (raw[(size_t)y * stride + (bit >> 3)] >> (8 - dp - (bit & 7))) &
                              ((1 << dp) - 1);
                if (3 * p + 2 >= desc->palette_len) {
                    set_error("palette index %d out of range at (%d, %d)", p, x, y);
                    return SV_ERR_PARAM;
                }
            }
    }
    return SV_OK;
}

int sv_image_decode_batch(int n, const uint8_t *const *data, const size_t *sizes,
                          uint8_t *const *raw, const size_t *raw_bytes, sv_raw_image *descs,
                          int *status, int threads) {
    if (n < 0 || (n > 0 && (!data || !sizes || !raw || !raw_bytes || !descs))) {
        set_error("NULL argument");
        return SV_ERR_NULL;
    }
    if (n == 0) return SV_OK;
    const int nt = std::max(1, std::min(threads > 0 ? threads : 1, n));
    std::vector<int> st((size_t)n, SV_OK);
    std::vector<std::string> msg((size_t)n);
    std::atomic<int> next{0};
    auto work = [&]() {
        for (int i; (i = next.fetch_add(1)) < n;) {
            st[i] = sv_image_decode_raw(data[i], sizes[i], raw[i], raw_bytes[i], &descs[i]);
            if (st[i] != SV_OK) msg[i] = sv_last_error();   // this thread's message
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < nt; ++t) pool.emplace_back(work);
    work();
    for (auto &t : pool) t.join();
    int rc = SV_OK;
    for (int i = 0; i < n; ++i) {
        if (status) status[i] = st[i];
        if (st[i] != SV_OK && rc == SV_OK) {
            rc = st[i];
            set_error("file %d: %s", i, msg[i].c_str());
        }
    }
    return rc;
}

int sv_raw_to_float(const uint8_t *raw, const sv_raw_image *desc, double *gray, double *rgb,
                    void *stream) {
    if (!raw || !desc || (!gray && !rgb)) { set_error("NULL argument"); return SV_ERR_NULL; }
    if (desc->width < 1 || desc->height < 1) { set_error("bad image size"); return SV_ERR_SHAPE; }
    const long npix = (long)desc->width * desc->height;
    count_launch();
    k_raw_to_float<<<(unsigned)((npix + 255) / 256), 256, 0, (cudaStream_t)stream>>>(raw, *desc,
                                                                                    gray, rgb);
    SV_LAUNCH_CHECK();
    return SV_OK;
}

}  // extern "C"
