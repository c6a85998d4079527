// grb_zstd.c: decoder of the Zstandard frame format (RFC 8878), host code.
//
// The reference compresses each block of a serialized matrix's arrays as one
// Zstandard frame (its default method, Source/serialize/GB_serialize_array.c
// through Source/zstd_wrapper), with the zstd library it vendors.  This file
// restates the published format's decoding steps in its own code: frame and
// block headers, raw / RLE / compressed blocks, the literals section (raw,
// RLE, Huffman with one or four streams, repeated tables), the sequences
// section (predefined, RLE, FSE-coded and repeated tables for literal
// lengths, match lengths and offsets), repeat offsets, and sequence
// execution.  Dictionaries are not supported (the reference uses none); a
// content checksum is skipped, not verified.  Every read is bounds-checked:
// a malformed frame gives -1, never a read or write outside the buffers.

#include <stdint.h>
#include <stdbool.h>
#include <stdlib.h>
#include <string.h>

#define HIDDEN __attribute__((visibility("hidden")))
#define MAX_BLOCK (128 * 1024)

static inline int highbit(uint32_t x) { return 31 - __builtin_clz(x); }

static inline uint32_t le16(const uint8_t *p) { return (uint32_t)p[0] | ((uint32_t)p[1] << 8); }
static inline uint32_t le24(const uint8_t *p) { return le16(p) | ((uint32_t)p[2] << 16); }
static inline uint32_t le32(const uint8_t *p) { return le24(p) | ((uint32_t)p[3] << 24); }

//------------------------------------------------------------------------------
// bit readers
//------------------------------------------------------------------------------

// bits [lo, lo+n) of a little-endian byte string of len bytes, zero beyond
// either end (n <= 56)
static inline uint64_t bits_at(const uint8_t *p, int64_t len, int64_t lo, int n)
{
    if (n == 0) return 0;
    if (lo < 0)
    {
        const int k = n + (int)lo;
        if (k <= 0) return 0;
        return bits_at(p, len, 0, k) << (-lo);
    }
    const int64_t byte = lo >> 3;
    uint64_t w = 0;
    if (byte < len) memcpy(&w, p + byte, (size_t)(len - byte < 8 ? len - byte : 8));
    return (w >> (lo & 7)) & ((1ull << n) - 1);
}

// backward stream: read from the last bit down; the highest set bit of the
// last byte marks the start
typedef struct { const uint8_t *p; int64_t len, bit; } bwd_t;

static bool bwd_init(bwd_t *b, const uint8_t *p, int64_t len)
{
    if (len <= 0 || p[len - 1] == 0) return false;
    b->p = p;
    b->len = len;
    b->bit = 8 * (len - 1) + highbit(p[len - 1]);
    return true;
}

static inline uint64_t bwd_read(bwd_t *b, int n)
{
    b->bit -= n;
    return bits_at(b->p, b->len, b->bit, n);
}

static inline uint64_t bwd_peek(const bwd_t *b, int n)
{
    return bits_at(b->p, b->len, b->bit - n, n);
}

//------------------------------------------------------------------------------
// FSE tables
//------------------------------------------------------------------------------

typedef struct { uint8_t sym, nb; uint16_t base; } fse_cell;
typedef struct { int al; bool ok; fse_cell cell[1 << 9]; } fse_table;

// normalized counts from a forward bit string (the FSE table description);
// returns the bytes it used, or -1
static int64_t fse_counts(const uint8_t *src, int64_t slen, int max_al, int max_sym,
                          int16_t *norm, int *nsym, int *al_out)
{
    int64_t pos = 0;
    const int al = (int)bits_at(src, slen, pos, 4) + 5;
    pos += 4;
    if (al > max_al) return -1;
    int remaining = (1 << al) + 1, threshold = 1 << al, nb = al + 1, s = 0;
    bool prev0 = false;
    while (remaining > 1 && s <= max_sym)
    {
        if (prev0)
        {
            int r;
            do
            {
                r = (int)bits_at(src, slen, pos, 2);
                pos += 2;
                for (int k = 0; k < r; k++)
                {
                    if (s > max_sym) return -1;
                    norm[s++] = 0;
                }
            } while (r == 3);
            if (s > max_sym) return -1;
        }
        const int max = (2 * threshold - 1) - remaining;
        const int v = (int)bits_at(src, slen, pos, nb);
        int count;
        if ((v & (threshold - 1)) < max)
        {
            count = v & (threshold - 1);
            pos += nb - 1;
        }
        else
        {
            count = v & (2 * threshold - 1);
            if (count >= threshold) count -= max;
            pos += nb;
        }
        count--;
        remaining -= count < 0 ? -count : count;
        if (remaining < 1) return -1;
        norm[s++] = (int16_t)count;
        prev0 = (count == 0);
        while (remaining < threshold)
        {
            nb--;
            threshold >>= 1;
        }
    }
    if (remaining != 1 || pos > 8 * slen) return -1;
    *nsym = s;
    *al_out = al;
    return (pos + 7) / 8;
}

// decoding table of the normalized counts: symbols of probability "less than
// one" at the top, the rest spread with the format's step, then each cell's
// bit count and next-state base
static bool fse_build(fse_table *t, const int16_t *norm, int nsym, int al)
{
    const int size = 1 << al;
    int high = size - 1;
    uint16_t next[256];
    for (int s = 0; s < nsym; s++)
    {
        if (norm[s] == -1)
        {
            if (high < 0) return false;
            t->cell[high--].sym = (uint8_t)s;
            next[s] = 1;
        }
        else
        {
            if (norm[s] < 0) return false;
            next[s] = (uint16_t)norm[s];
        }
    }
    const int step = (size >> 1) + (size >> 3) + 3, mask = size - 1;
    int pos = 0;
    for (int s = 0; s < nsym; s++)
        for (int k = 0; k < norm[s]; k++)
        {
            t->cell[pos].sym = (uint8_t)s;
            do pos = (pos + step) & mask; while (pos > high);
        }
    if (pos != 0) return false;
    for (int u = 0; u < size; u++)
    {
        const int s = t->cell[u].sym;
        const uint32_t x = next[s]++;
        if (x == 0) return false;
        const int nb = al - highbit(x);
        t->cell[u].nb = (uint8_t)nb;
        t->cell[u].base = (uint16_t)((x << nb) - (uint32_t)size);
    }
    t->al = al;
    t->ok = true;
    return true;
}

static void fse_rle(fse_table *t, uint8_t sym)
{
    t->al = 0;
    t->cell[0].sym = sym;
    t->cell[0].nb = 0;
    t->cell[0].base = 0;
    t->ok = true;
}

// the format's predefined distributions (RFC 8878 section 3.1.1.3.2.2)
static const int16_t LL_DEFAULT[36] = {
    4, 3, 2, 2, 2, 2, 2, 2, 2, 2, 2, 2, 2, 1, 1, 1,
    2, 2, 2, 2, 2, 2, 2, 2, 2, 3, 2, 1, 1, 1, 1, 1, -1, -1, -1, -1};
static const int16_t ML_DEFAULT[53] = {
    1, 4, 3, 2, 2, 2, 2, 2, 2, 1, 1, 1, 1, 1, 1, 1,
    1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1,
    1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, -1, -1,
    -1, -1, -1, -1, -1};
static const int16_t OF_DEFAULT[29] = {
    1, 1, 1, 1, 1, 1, 2, 2, 2, 1, 1, 1, 1, 1, 1, 1,
    1, 1, 1, 1, 1, 1, 1, 1, -1, -1, -1, -1, -1};

// literal-length and match-length codes: baseline and extra bits
static const uint32_t LL_BASE[36] = {
    0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15,
    16, 18, 20, 22, 24, 28, 32, 40, 48, 64, 128, 256, 512, 1024, 2048, 4096,
    8192, 16384, 32768, 65536};
static const uint8_t LL_BITS[36] = {
    0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0,
    1, 1, 1, 1, 2, 2, 3, 3, 4, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16};
static const uint32_t ML_BASE[53] = {
    3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16, 17, 18,
    19, 20, 21, 22, 23, 24, 25, 26, 27, 28, 29, 30, 31, 32, 33, 34,
    35, 37, 39, 41, 43, 47, 51, 59, 67, 83, 99, 131, 259, 515, 1027, 2051,
    4099, 8195, 16387, 32771, 65539};
static const uint8_t ML_BITS[53] = {
    0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0,
    0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0,
    1, 1, 1, 1, 2, 2, 3, 3, 4, 4, 5, 7, 8, 9, 10, 11,
    12, 13, 14, 15, 16};

//------------------------------------------------------------------------------
// Huffman tables
//------------------------------------------------------------------------------

typedef struct { uint8_t sym, nb; } huf_cell;
typedef struct { int maxbits; bool ok; huf_cell cell[1 << 11]; } huf_table;

// the Huffman tree description (weights direct or FSE-coded); returns bytes
// used or -1
static int64_t huf_read(huf_table *h, const uint8_t *src, int64_t slen)
{
    uint8_t w[256];
    int n = 0;
    int64_t used;
    if (slen < 1) return -1;
    const int hb = src[0];
    if (hb >= 128)
    {
        n = hb - 127;
        used = 1 + (n + 1) / 2;
        if (used > slen) return -1;
        for (int k = 0; k < n; k++)
        {
            const uint8_t byte = src[1 + k / 2];
            w[k] = (k & 1) ? (byte & 15) : (byte >> 4);
        }
    }
    else
    {
        used = 1 + hb;
        if (hb == 0 || used > slen) return -1;
        int16_t norm[256];
        int nsym, al;
        const int64_t c = fse_counts(src + 1, hb, 6, 255, norm, &nsym, &al);
        if (c < 0 || c >= hb) return -1;
        fse_table t;
        if (!fse_build(&t, norm, nsym, al)) return -1;
        bwd_t b;
        if (!bwd_init(&b, src + 1 + c, hb - c)) return -1;
        uint32_t s1 = (uint32_t)bwd_read(&b, al), s2 = (uint32_t)bwd_read(&b, al);
        // two interleaved states; the stream running out ends the list
        // (at most 255 weights: the implied last one makes 256 symbols)
        for (;;)
        {
            if (n >= 255) return -1;
            w[n++] = t.cell[s1].sym;
            s1 = t.cell[s1].base + (uint32_t)bwd_read(&b, t.cell[s1].nb);
            if (n >= 255) return -1;
            if (b.bit < 0) { w[n++] = t.cell[s2].sym; break; }
            w[n++] = t.cell[s2].sym;
            s2 = t.cell[s2].base + (uint32_t)bwd_read(&b, t.cell[s2].nb);
            if (n >= 255) return -1;
            if (b.bit < 0) { w[n++] = t.cell[s1].sym; break; }
        }
    }
    // the last symbol's weight completes the sum to a power of two
    uint32_t total = 0;
    int count[13] = {0};
    for (int k = 0; k < n; k++)
    {
        if (w[k] > 11) return -1;
        if (w[k]) total += 1u << (w[k] - 1);
        count[w[k]]++;
    }
    if (total == 0) return -1;
    const int maxbits = highbit(total) + 1;
    if (maxbits > 11) return -1;
    const uint32_t rest = (1u << maxbits) - total;
    if (rest == 0 || (rest & (rest - 1))) return -1;
    w[n] = (uint8_t)(highbit(rest) + 1);
    count[w[n]]++;
    n++;
    // canonical codes: lowest weights (longest codes) first, symbols in order
    uint32_t start[13];
    start[1] = 0;
    for (int k = 1; k < 12; k++) start[k + 1] = start[k] + ((uint32_t)count[k] << (k - 1));
    for (int s = 0; s < n; s++)
    {
        if (!w[s]) continue;
        const uint32_t len = 1u << (w[s] - 1);
        const uint8_t nb = (uint8_t)(maxbits + 1 - w[s]);
        for (uint32_t q = 0; q < len; q++)
        {
            h->cell[start[w[s]] + q].sym = (uint8_t)s;
            h->cell[start[w[s]] + q].nb = nb;
        }
        start[w[s]] += len;
    }
    h->maxbits = maxbits;
    h->ok = true;
    return used;
}

static bool huf_stream(const huf_table *h, const uint8_t *src, int64_t slen, uint8_t *dst,
                       int64_t n)
{
    bwd_t b;
    if (!bwd_init(&b, src, slen)) return false;
    for (int64_t k = 0; k < n; k++)
    {
        const huf_cell c = h->cell[bwd_peek(&b, h->maxbits)];
        dst[k] = c.sym;
        b.bit -= c.nb;
    }
    return b.bit == 0;
}

//------------------------------------------------------------------------------
// blocks
//------------------------------------------------------------------------------

typedef struct
{
    huf_table huf;
    fse_table ll, of, ml;
    uint32_t rep[3];
    uint8_t lit[MAX_BLOCK];
} zctx;

// the literals section; returns bytes used or -1
static int64_t literals(zctx *z, const uint8_t *src, int64_t slen, int64_t *nlit)
{
    if (slen < 1) return -1;
    const int type = src[0] & 3, sf = (src[0] >> 2) & 3;
    if (type <= 1)
    {
        int64_t hs, size;
        if (sf == 0 || sf == 2) { hs = 1; size = src[0] >> 3; }
        else if (sf == 1) { if (slen < 2) return -1; hs = 2; size = (src[0] >> 4) + ((int64_t)src[1] << 4); }
        else { if (slen < 3) return -1; hs = 3; size = (src[0] >> 4) + ((int64_t)src[1] << 4) + ((int64_t)src[2] << 12); }
        if (size > MAX_BLOCK) return -1;
        *nlit = size;
        if (type == 0)
        {
            if (hs + size > slen) return -1;
            memcpy(z->lit, src + hs, (size_t)size);
            return hs + size;
        }
        if (hs + 1 > slen) return -1;
        memset(z->lit, src[hs], (size_t)size);
        return hs + 1;
    }
    int64_t hs, regen, comp;
    int nstreams = sf == 0 ? 1 : 4;
    if (sf <= 1)
    {
        if (slen < 3) return -1;
        const uint32_t h = le24(src);
        hs = 3; regen = (h >> 4) & 0x3FF; comp = (h >> 14) & 0x3FF;
    }
    else if (sf == 2)
    {
        if (slen < 4) return -1;
        const uint32_t h = le32(src);
        hs = 4; regen = (h >> 4) & 0x3FFF; comp = (h >> 18) & 0x3FFF;
    }
    else
    {
        if (slen < 5) return -1;
        const uint64_t h = le32(src) | ((uint64_t)src[4] << 32);
        hs = 5; regen = (int64_t)((h >> 4) & 0x3FFFF); comp = (int64_t)((h >> 22) & 0x3FFFF);
    }
    if (regen > MAX_BLOCK || hs + comp > slen) return -1;
    const uint8_t *p = src + hs;
    int64_t rem = comp;
    if (type == 2)
    {
        const int64_t used = huf_read(&z->huf, p, rem);
        if (used < 0) { z->huf.ok = false; return -1; }
        p += used;
        rem -= used;
    }
    else if (!z->huf.ok)
    {
        return -1;                                  // treeless without a table
    }
    if (nstreams == 1)
    {
        if (!huf_stream(&z->huf, p, rem, z->lit, regen)) return -1;
    }
    else
    {
        if (rem < 6) return -1;
        const int64_t l1 = le16(p), l2 = le16(p + 2), l3 = le16(p + 4);
        const int64_t l4 = rem - 6 - l1 - l2 - l3;
        const int64_t seg = (regen + 3) / 4, last = regen - 3 * seg;
        if (l4 < 1 || last < 0) return -1;
        const uint8_t *q = p + 6;
        if (!huf_stream(&z->huf, q, l1, z->lit, seg) ||
            !huf_stream(&z->huf, q + l1, l2, z->lit + seg, seg) ||
            !huf_stream(&z->huf, q + l1 + l2, l3, z->lit + 2 * seg, seg) ||
            !huf_stream(&z->huf, q + l1 + l2 + l3, l4, z->lit + 3 * seg, last))
            return -1;
    }
    *nlit = regen;
    return hs + comp;
}

// one table of the sequences section by its mode; returns bytes used or -1
static int64_t seq_table(fse_table *t, int mode, const uint8_t *src, int64_t slen,
                         const int16_t *def, int ndef, int def_al, int max_al, int max_sym)
{
    if (mode == 0)
        return fse_build(t, def, ndef, def_al) ? 0 : -1;
    if (mode == 1)
    {
        if (slen < 1 || src[0] > max_sym) return -1;
        fse_rle(t, src[0]);
        return 1;
    }
    if (mode == 2)
    {
        int16_t norm[64];
        int nsym, al;
        const int64_t c = fse_counts(src, slen, max_al, max_sym, norm, &nsym, &al);
        if (c < 0 || !fse_build(t, norm, nsym, al)) { t->ok = false; return -1; }
        return c;
    }
    return t->ok ? 0 : -1;                          // repeat the previous table
}

static bool block(zctx *z, const uint8_t *src, int64_t slen, uint8_t *dst, int64_t *op_io,
                  int64_t dlen, int64_t frame_start)
{
    int64_t nlit = 0;
    const int64_t lused = literals(z, src, slen, &nlit);
    if (lused < 0) return false;
    const uint8_t *p = src + lused;
    int64_t rem = slen - lused;
    if (rem < 1) return false;
    int64_t nseq;
    if (p[0] < 128) { nseq = p[0]; p += 1; rem -= 1; }
    else if (p[0] < 255) { if (rem < 2) return false; nseq = ((int64_t)(p[0] - 128) << 8) + p[1]; p += 2; rem -= 2; }
    else { if (rem < 3) return false; nseq = p[1] + ((int64_t)p[2] << 8) + 0x7F00; p += 3; rem -= 3; }
    int64_t op = *op_io, lp = 0;
    if (nseq > 0)
    {
        if (rem < 1) return false;
        const int modes = p[0];
        p += 1;
        rem -= 1;
        if (modes & 3) return false;
        int64_t u;
        if ((u = seq_table(&z->ll, (modes >> 6) & 3, p, rem, LL_DEFAULT, 36, 6, 9, 35)) < 0) return false;
        p += u; rem -= u;
        if ((u = seq_table(&z->of, (modes >> 4) & 3, p, rem, OF_DEFAULT, 29, 5, 8, 31)) < 0) return false;
        p += u; rem -= u;
        if ((u = seq_table(&z->ml, (modes >> 2) & 3, p, rem, ML_DEFAULT, 53, 6, 9, 52)) < 0) return false;
        p += u; rem -= u;
        bwd_t b;
        if (!bwd_init(&b, p, rem)) return false;
        uint32_t ls = (uint32_t)bwd_read(&b, z->ll.al);
        uint32_t os = (uint32_t)bwd_read(&b, z->of.al);
        uint32_t ms = (uint32_t)bwd_read(&b, z->ml.al);
        for (int64_t k = 0; k < nseq; k++)
        {
            const int oc = z->of.cell[os].sym, mc = z->ml.cell[ms].sym, lc = z->ll.cell[ls].sym;
            if (oc > 31 || mc > 52 || lc > 35) return false;
            const uint64_t ov = (1ull << oc) + bwd_read(&b, oc);
            const int64_t ml = ML_BASE[mc] + (int64_t)bwd_read(&b, ML_BITS[mc]);
            const int64_t ll = LL_BASE[lc] + (int64_t)bwd_read(&b, LL_BITS[lc]);
            uint64_t off;
            if (ov > 3)
            {
                off = ov - 3;
                z->rep[2] = z->rep[1];
                z->rep[1] = z->rep[0];
                z->rep[0] = (uint32_t)off;
            }
            else
            {
                const int idx = (int)ov - 1 + (ll == 0 ? 1 : 0);
                if (idx == 0) off = z->rep[0];
                else
                {
                    off = idx == 3 ? (uint64_t)z->rep[0] - 1 : z->rep[idx];
                    if (idx > 1) z->rep[2] = z->rep[1];
                    z->rep[1] = z->rep[0];
                    z->rep[0] = (uint32_t)off;
                }
            }
            if (k + 1 < nseq)
            {
                ls = z->ll.cell[ls].base + (uint32_t)bwd_read(&b, z->ll.cell[ls].nb);
                ms = z->ml.cell[ms].base + (uint32_t)bwd_read(&b, z->ml.cell[ms].nb);
                os = z->of.cell[os].base + (uint32_t)bwd_read(&b, z->of.cell[os].nb);
            }
            // execute: ll literals, then ml bytes from off back
            if (ll > nlit - lp || ll > dlen - op) return false;
            memcpy(dst + op, z->lit + lp, (size_t)ll);
            op += ll;
            lp += ll;
            if (off == 0 || (int64_t)off > op - frame_start || ml > dlen - op) return false;
            uint8_t *d = dst + op;
            const uint8_t *s = d - off;
            if ((int64_t)off >= ml) memcpy(d, s, (size_t)ml);
            else for (int64_t q = 0; q < ml; q++) d[q] = s[q];
            op += ml;
        }
        if (b.bit != 0) return false;
    }
    else if (rem != 0)
    {
        return false;
    }
    // the literals after the last sequence
    if (nlit - lp > dlen - op) return false;
    memcpy(dst + op, z->lit + lp, (size_t)(nlit - lp));
    op += nlit - lp;
    *op_io = op;
    return true;
}

//------------------------------------------------------------------------------
// frames
//------------------------------------------------------------------------------

static int64_t frames(zctx *z, const uint8_t *src, int64_t slen, uint8_t *dst, int64_t dlen);

// Decode the frames in src[0..slen) into dst (room dlen).  Returns the bytes
// written, or -1 for a malformed or unsupported frame.
HIDDEN int64_t grb_zstd_decode(const uint8_t *src, int64_t slen, uint8_t *dst, int64_t dlen)
{
    zctx *zp = malloc(sizeof(zctx));
    if (!zp) return -1;
    const int64_t r = frames(zp, src, slen, dst, dlen);
    free(zp);
    return r;
}

static int64_t frames(zctx *zp, const uint8_t *src, int64_t slen, uint8_t *dst, int64_t dlen)
{
    zctx *const z = zp;
    int64_t ip = 0, op = 0;
    while (ip < slen)
    {
        if (slen - ip < 4) return -1;
        const uint32_t magic = le32(src + ip);
        if ((magic & 0xFFFFFFF0u) == 0x184D2A50u)  // skippable frame
        {
            if (slen - ip < 8) return -1;
            const int64_t size = le32(src + ip + 4);
            if (size > slen - ip - 8) return -1;
            ip += 8 + size;
            continue;
        }
        if (magic != 0xFD2FB528u) return -1;
        ip += 4;
        if (ip >= slen) return -1;
        const int fhd = src[ip++];
        const int fcs_flag = fhd >> 6, single = (fhd >> 5) & 1, checksum = (fhd >> 2) & 1;
        const int did_flag = fhd & 3;
        if (fhd & 8) return -1;                     // reserved bit
        if (!single) ip++;                          // window descriptor
        static const int DID_SIZE[4] = {0, 1, 2, 4};
        const int did_size = DID_SIZE[did_flag];
        const int fcs_size = fcs_flag == 0 ? single : (fcs_flag == 1 ? 2 : (fcs_flag == 2 ? 4 : 8));
        if (ip + did_size + fcs_size > slen) return -1;
        uint32_t did = 0;
        for (int k = 0; k < did_size; k++) did |= (uint32_t)src[ip + k] << (8 * k);
        if (did != 0) return -1;                    // dictionaries unsupported
        ip += did_size;
        int64_t fcs = -1;
        if (fcs_size > 0)
        {
            uint64_t v = 0;
            for (int k = 0; k < fcs_size; k++) v |= (uint64_t)src[ip + k] << (8 * k);
            if (fcs_size == 2) v += 256;
            fcs = (int64_t)v;
            ip += fcs_size;
        }
        const int64_t frame_start = op;
        z->huf.ok = false;
        z->ll.ok = z->of.ok = z->ml.ok = false;
        z->rep[0] = 1; z->rep[1] = 4; z->rep[2] = 8;
        for (;;)
        {
            if (slen - ip < 3) return -1;
            const uint32_t bh = le24(src + ip);
            ip += 3;
            const int last = bh & 1, type = (bh >> 1) & 3;
            const int64_t size = bh >> 3;
            if (size > MAX_BLOCK) return -1;
            if (type == 0)
            {
                if (size > slen - ip || size > dlen - op) return -1;
                memcpy(dst + op, src + ip, (size_t)size);
                ip += size;
                op += size;
            }
            else if (type == 1)
            {
                if (ip >= slen || size > dlen - op) return -1;
                memset(dst + op, src[ip], (size_t)size);
                ip += 1;
                op += size;
            }
            else if (type == 2)
            {
                if (size > slen - ip) return -1;
                if (!block(z, src + ip, size, dst, &op, dlen, frame_start)) return -1;
                ip += size;
            }
            else
            {
                return -1;
            }
            if (last) break;
        }
        if (checksum)
        {
            if (slen - ip < 4) return -1;
            ip += 4;
        }
        if (fcs >= 0 && op - frame_start != fcs) return -1;
    }
    return op;
}
