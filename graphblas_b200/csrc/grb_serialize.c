// grb_serialize.c: the reference's serialized-matrix blob (GxB_Matrix_serialize
// / GxB_Matrix_deserialize, Source/serialize/GB_serialize.c:43 and
// GB_deserialize.c:22), read and written on the host so that graphs saved by
// the reference can be loaded into HBM and graphs computed here can be read
// back by it.
//
// Blob layout (all fields little-endian, in this order; GB_serialize.c:300-360):
//   uint64 blob_size; int32 typecode, version;
//   int64 vlen, vdim, nvec, nvec_nonempty, nvals, typesize;
//   int64 Ap_len, Ah_len, Ab_len, Ai_len, Ax_len   (bytes of each array);
//   float hyper_switch, bitmap_switch; int32 sparsity_control,
//   int32 sparsity_iso_csc = 4*sparsity + 2*iso + is_csc;
//   int32 (nblocks, method) for Ap, Ah, Ab, Ai, Ax;
//   [user-defined type name, 128 bytes, only for the user-defined type code];
//   int64 cumulative compressed block ends, nblocks per array, same order;
//   the compressed blocks of Ap, Ah, Ab, Ai, Ax;
//   the matrix name and the element-type name, each nul-terminated.
// Each array of len bytes is cut into nblocks equal parts (the reference's
// GB_PARTITION rule, floating-point split points) compressed one by one.
//
// Compression methods read: none (-1 / len < 256 stored raw), LZ4 (1000) and
// LZ4HC (2000), both decoded with the LZ4 block format below, and ZSTD (3000,
// and 0, the reference's default), decoded by grb_zstd.c.
// Blobs written here are uncompressed and sparse, by row (by column for
// vectors), which the reference reads.  Types: the built-in types of this
// library (bool, int32, uint32, int64, uint64, fp32, fp64).  All four
// sparsity forms are read; they come back as CSR by row.

#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <stdbool.h>
#include "grb_b200.h"

enum { S_SUCCESS = 0, S_NULL = -2, S_INVALID_VALUE = -3, S_DOMAIN = -5,
       S_NOT_IMPLEMENTED = -8, S_OUT_OF_MEMORY = -102, S_INSUFFICIENT = -103,
       S_INVALID_OBJECT = -104 };

enum { HYPER = 1, SPARSE = 2, BITMAP = 4, FULL = 8 };
enum { M_NONE = -1, M_LZ4 = 1000, M_LZ4HC = 2000, M_ZSTD = 3000 };

// Zstandard frame decoder (grb_zstd.c)
int64_t grb_zstd_decode(const uint8_t *src, int64_t slen, uint8_t *dst, int64_t dlen);

#define HEADER_SIZE (8 + 11 * 8 + 14 * 4 + 2 * 4)
#define UDT_CODE 14
#define NAME_LEN 128
#define VERSION_9_3_1 9003001

static size_t type_bytes(int code)
{
    switch (code)
    {
        case 1: return 1;
        case 6: case 7: case 10: return 4;
        case 8: case 9: case 11: return 8;
    }
    return 0;
}

static const char *type_name(int code)
{
    switch (code)
    {
        case 1: return "GrB_BOOL";
        case 6: return "GrB_INT32";
        case 7: return "GrB_UINT32";
        case 8: return "GrB_INT64";
        case 9: return "GrB_UINT64";
        case 10: return "GrB_FP32";
        case 11: return "GrB_FP64";
    }
    return "";
}

//------------------------------------------------------------------------------
// LZ4 block format (the published format: a token whose high nibble is the
// literal count and low nibble the match length - 4, each extended by bytes
// of 255 when 15, the literals, a 2-byte little-endian back offset, and a
// final sequence of literals only).  Returns the decoded size or -1.
//------------------------------------------------------------------------------

static int64_t lz4_decode(const uint8_t *src, int64_t slen, uint8_t *dst, int64_t dlen)
{
    int64_t ip = 0, op = 0;
    while (ip < slen)
    {
        const uint8_t token = src[ip++];
        int64_t lit = token >> 4;
        if (lit == 15)
        {
            uint8_t b;
            do
            {
                if (ip >= slen) return -1;
                b = src[ip++];
                lit += b;
            } while (b == 255);
        }
        if (lit > slen - ip || lit > dlen - op) return -1;
        memcpy(dst + op, src + ip, (size_t)lit);
        ip += lit;
        op += lit;
        if (ip == slen) break;                  // the last sequence
        if (slen - ip < 2) return -1;
        const int64_t off = (int64_t)src[ip] | ((int64_t)src[ip + 1] << 8);
        ip += 2;
        if (off == 0 || off > op) return -1;
        int64_t mlen = (token & 15);
        if (mlen == 15)
        {
            uint8_t b;
            do
            {
                if (ip >= slen) return -1;
                b = src[ip++];
                mlen += b;
            } while (b == 255);
        }
        mlen += 4;
        if (mlen > dlen - op) return -1;
        // byte by byte: the match may overlap the bytes it produces
        for (int64_t q = 0; q < mlen; q++, op++) dst[op] = dst[op - off];
    }
    return op;
}

//------------------------------------------------------------------------------
// one array of the blob
//------------------------------------------------------------------------------

// start of block b of a len-byte array cut into n blocks (GB_PARTITION)
static int64_t part(int64_t b, int64_t len, int64_t n)
{
    if (b == 0) return 0;
    if (b == n) return len;
    return (int64_t)(((double)b * (double)len) / (double)n);
}

// read an array of len bytes compressed in nblocks blocks whose cumulative
// ends are ends[0..nblocks-1], starting at blob offset *s
static int read_array(const uint8_t *blob, size_t size, size_t *s, int64_t len,
                      int32_t nblocks, int32_t method, const uint8_t *ends_raw,
                      uint8_t **out)
{
    *out = NULL;
    if (len < 0 || nblocks < 0) return S_INVALID_OBJECT;
    if (len == 0)
    {
        if (nblocks > 0)
        {
            int64_t e;
            memcpy(&e, ends_raw + 8 * (nblocks - 1), 8);
            if (e < 0 || *s + (size_t)e > size) return S_INVALID_OBJECT;
            *s += (size_t)e;
        }
        return S_SUCCESS;
    }
    uint8_t *X = malloc((size_t)len);
    if (!X) return S_OUT_OF_MEMORY;
    const int32_t algo = method < 0 ? M_NONE : 1000 * (method / 1000);
    int rc = S_SUCCESS;
    int64_t total = 0;
    if (algo == M_NONE)
    {
        int64_t e = -1;
        if (nblocks == 1) memcpy(&e, ends_raw, 8);
        if (nblocks != 1 || e != len || *s + (size_t)len > size) rc = S_INVALID_OBJECT;
        else { memcpy(X, blob + *s, (size_t)len); total = len; }
    }
    else
    {
        // LZ4 / LZ4HC blocks, or ZSTD frames (any other method: the reference
        // maps every other value to ZSTD, GB_serialize_method.c); the blocks
        // decode independently, in parallel as the reference does
        // (Source/serialize/GB_deserialize_from_blob.c:100-175)
        const bool lz4 = (algo == M_LZ4 || algo == M_LZ4HC);
        bool ok = true;
        #pragma omp parallel for schedule(dynamic) reduction(&&:ok)
        for (int32_t b = 0; b < nblocks; b++)
        {
            int64_t s0 = 0, s1;
            if (b > 0) memcpy(&s0, ends_raw + 8 * (b - 1), 8);
            memcpy(&s1, ends_raw + 8 * b, 8);
            const int64_t k0 = part(b, len, nblocks), k1 = part(b + 1, len, nblocks);
            if (s0 < 0 || s1 <= s0 || k1 <= k0 || *s + (size_t)s1 > size)
                ok = false;
            else if (lz4)
                ok = lz4_decode(blob + *s + s0, s1 - s0, X + k0, k1 - k0) == k1 - k0;
            else
                ok = grb_zstd_decode(blob + *s + s0, s1 - s0, X + k0, k1 - k0) == k1 - k0;
        }
        if (!ok || nblocks == 0) rc = S_INVALID_OBJECT;
        else memcpy(&total, ends_raw + 8 * (nblocks - 1), 8);
    }
    if (rc != S_SUCCESS) { free(X); return rc; }
    *s += (size_t)(algo == M_NONE ? len : total);
    *out = X;
    return S_SUCCESS;
}

//------------------------------------------------------------------------------
// decode
//------------------------------------------------------------------------------

// a * b for a, b >= 0, or -1 when it overflows
static int64_t mul_or_neg(int64_t a, int64_t b)
{
    if (a == 0 || b == 0) return 0;
    return a > INT64_MAX / b ? -1 : a * b;
}

// the array lengths that the header's shape implies (GB_serialize.c:166-187),
// checked before any array is allocated
static bool lengths_ok(int sparsity, int64_t vlen, int64_t vdim, int64_t nvec, bool iso,
                       int64_t ts, const int64_t len[5])
{
    for (int a = 0; a < 5; a++) if (len[a] < 0) return false;
    if (sparsity == SPARSE || sparsity == HYPER)
    {
        const int64_t np = sparsity == SPARSE ? vdim : nvec;
        if (np >= INT64_MAX / 8 || len[0] != 8 * (np + 1) || len[2] != 0) return false;
        if (len[1] != (sparsity == HYPER ? 8 * nvec : 0)) return false;
        if (len[3] % 8) return false;
        return len[4] == mul_or_neg(ts, iso ? 1 : len[3] / 8);
    }
    if (sparsity == BITMAP || sparsity == FULL)
    {
        const int64_t held = mul_or_neg(vlen, vdim);
        if (held < 0 || len[0] != 0 || len[1] != 0 || len[3] != 0) return false;
        if (len[2] != (sparsity == BITMAP ? held : 0)) return false;
        return len[4] == mul_or_neg(ts, iso ? 1 : held);
    }
    return false;
}

int grb_b200_blob_decode(const void *blob_in, size_t blob_size, int expected_type,
                         int64_t *nrows, int64_t *ncols, int *type, int64_t **Cp,
                         int64_t **Ci, void **Cx, bool *iso_out)
{
    if (!blob_in || !nrows || !ncols || !type || !Cp || !Ci || !Cx) return S_NULL;
    *Cp = NULL; *Ci = NULL; *Cx = NULL;
    const uint8_t *blob = (const uint8_t *)blob_in;
    if (blob_size < HEADER_SIZE) return S_INVALID_OBJECT;
    size_t s = 0;
    #define RD(x, T) T x; memcpy(&x, blob + s, sizeof(T)); s += sizeof(T)
    RD(size2, uint64_t);
    RD(typecode, int32_t);
    if (size2 != (uint64_t)blob_size || typecode < 1 || typecode > UDT_CODE)
        return S_INVALID_OBJECT;
    RD(version, int32_t);
    RD(vlen, int64_t); RD(vdim, int64_t); RD(nvec, int64_t); RD(nvec_nonempty, int64_t);
    RD(nvals, int64_t); RD(typesize, int64_t);
    RD(p_len, int64_t); RD(h_len, int64_t); RD(b_len, int64_t); RD(i_len, int64_t);
    RD(x_len, int64_t);
    RD(hyper_switch, float); RD(bitmap_switch, float);
    RD(sparsity_control, int32_t); RD(sic, int32_t);
    int32_t nb[5], mt[5];
    for (int a = 0; a < 5; a++) { RD(n_, int32_t); RD(m_, int32_t); nb[a] = n_; mt[a] = m_; }
    #undef RD
    (void)version; (void)nvec_nonempty; (void)nvals; (void)hyper_switch;
    (void)bitmap_switch; (void)sparsity_control;
    const size_t ts = type_bytes(typecode);
    if (ts == 0) return typecode == UDT_CODE ? S_DOMAIN : S_NOT_IMPLEMENTED;
    if (expected_type != 0 && expected_type != typecode) return S_DOMAIN;
    if (typesize != (int64_t)ts) return S_DOMAIN;
    if (vlen < 0 || vdim < 0 || nvec < 0 || nvec > vdim) return S_INVALID_OBJECT;
    const int sparsity = sic / 4;
    const bool iso = (sic & 2) != 0, is_csc = (sic & 1) != 0;
    const int64_t lens[5] = {p_len, h_len, b_len, i_len, x_len};
    if (!lengths_ok(sparsity, vlen, vdim, nvec, iso, (int64_t)ts, lens)) return S_INVALID_OBJECT;
    // the block ends of the five arrays
    const uint8_t *ends[5];
    for (int a = 0; a < 5; a++)
    {
        if (nb[a] < 0 || s + 8 * (size_t)nb[a] > blob_size) return S_INVALID_OBJECT;
        ends[a] = blob + s;
        s += 8 * (size_t)nb[a];
    }
    uint8_t *P = NULL, *H = NULL, *B = NULL, *I = NULL, *X = NULL;
    uint8_t **dst[5] = {&P, &H, &B, &I, &X};
    int rc = S_SUCCESS;
    for (int a = 0; a < 5 && rc == S_SUCCESS; a++)
        rc = read_array(blob, blob_size, &s, lens[a], nb[a], mt[a], ends[a], dst[a]);
    // vectors of the stored form as (vector, index) pairs, by vector
    int64_t *vp = NULL, *vi = NULL;
    int64_t nnz = 0;
    if (rc == S_SUCCESS)
    {
        vp = calloc((size_t)vdim + 1, sizeof(int64_t));
        if (!vp) rc = S_OUT_OF_MEMORY;
    }
    if (rc == S_SUCCESS && (sparsity == SPARSE || sparsity == HYPER))
    {
        const int64_t *p = (const int64_t *)P, *h = (const int64_t *)H;
        const int64_t np = sparsity == SPARSE ? vdim : nvec;
        if (!P || p[0] != 0 || p[np] != i_len / 8) rc = S_INVALID_OBJECT;
        for (int64_t k = 0; rc == S_SUCCESS && k < np; k++)
        {
            const int64_t v = sparsity == SPARSE ? k : h[k];
            if (p[k + 1] < p[k] || v < 0 || v >= vdim || (k > 0 && sparsity == HYPER && h[k] <= h[k - 1]))
                rc = S_INVALID_OBJECT;
            else
                vp[v + 1] = p[k + 1] - p[k];
        }
        if (rc == S_SUCCESS)
        {
            nnz = p[np];
            for (int64_t v = 0; v < vdim; v++) vp[v + 1] += vp[v];
            vi = (int64_t *)I;
            I = NULL;
            // indices in range and strictly ascending in each vector (the
            // reference serializes only finished, unjumbled matrices)
            for (int64_t v = 0; rc == S_SUCCESS && v < vdim; v++)
                for (int64_t q = vp[v]; q < vp[v + 1]; q++)
                    if (vi[q] < 0 || vi[q] >= vlen || (q > vp[v] && vi[q] <= vi[q - 1]))
                    {
                        rc = S_INVALID_OBJECT;
                        break;
                    }
        }
    }
    else if (rc == S_SUCCESS && (sparsity == BITMAP || sparsity == FULL))
    {
        const int64_t held = vlen * vdim;           // no overflow: lengths_ok
        if (sparsity == BITMAP && held > 0 && !B) rc = S_INVALID_OBJECT;
        for (int64_t q = 0; rc == S_SUCCESS && q < held; q++)
            if (sparsity == FULL || B[q]) nnz++;
        if (rc == S_SUCCESS)
        {
            vi = malloc((size_t)(nnz ? nnz : 1) * sizeof(int64_t));
            if (!vi) rc = S_OUT_OF_MEMORY;
        }
        int64_t e = 0;
        for (int64_t v = 0; rc == S_SUCCESS && v < vdim; v++)
        {
            for (int64_t k = 0; k < vlen; k++)
                if (sparsity == FULL || B[v * vlen + k]) vi[e++] = k;
            vp[v + 1] = e;
        }
    }
    else if (rc == S_SUCCESS)
    {
        rc = S_INVALID_OBJECT;
    }
    // values in the stored order (one value when iso), gathered for bitmap
    char *vx = NULL;
    if (rc == S_SUCCESS)
    {
        const int64_t need = iso ? 1 : (sparsity == BITMAP || sparsity == FULL ? vlen * vdim : nnz);
        if ((need > 0 && !X) || x_len != (int64_t)ts * need) rc = S_INVALID_OBJECT;
    }
    if (rc == S_SUCCESS)
    {
        if (iso || sparsity != BITMAP)
        {
            vx = (char *)X;
            X = NULL;
        }
        else
        {
            vx = malloc((size_t)(nnz ? nnz : 1) * ts);
            if (!vx) rc = S_OUT_OF_MEMORY;
            int64_t e = 0;
            for (int64_t q = 0; rc == S_SUCCESS && q < vlen * vdim; q++)
                if (B[q]) memcpy(vx + e++ * ts, X + q * ts, ts);
        }
    }
    // by row: the stored vectors are rows; by column: transpose to rows
    if (rc == S_SUCCESS)
    {
        *nrows = is_csc ? vlen : vdim;
        *ncols = is_csc ? vdim : vlen;
        *type = typecode;
        if (iso_out) *iso_out = iso;
        if (!is_csc)
        {
            *Cp = vp; *Ci = vi; *Cx = vx;
            vp = NULL; vi = NULL; vx = NULL;
        }
        else
        {
            const int64_t m = vlen;
            int64_t *rp = calloc((size_t)m + 1, sizeof(int64_t));
            int64_t *ri = malloc((size_t)(nnz ? nnz : 1) * sizeof(int64_t));
            char *rx = iso ? NULL : malloc((size_t)(nnz ? nnz : 1) * ts);
            if (!rp || !ri || (!iso && !rx)) rc = S_OUT_OF_MEMORY;
            if (rc == S_SUCCESS)
            {
                for (int64_t q = 0; q < nnz; q++) rp[vi[q] + 1]++;
                for (int64_t r = 0; r < m; r++) rp[r + 1] += rp[r];
                int64_t *fill = malloc((size_t)(m ? m : 1) * sizeof(int64_t));
                if (!fill) rc = S_OUT_OF_MEMORY;
                else
                {
                    memcpy(fill, rp, (size_t)m * sizeof(int64_t));
                    // columns in ascending order, so each row comes out sorted
                    for (int64_t c = 0; c < vdim; c++)
                        for (int64_t q = vp[c]; q < vp[c + 1]; q++)
                        {
                            const int64_t d = fill[vi[q]]++;
                            ri[d] = c;
                            if (!iso) memcpy(rx + d * ts, vx + q * ts, ts);
                        }
                    free(fill);
                }
            }
            if (rc == S_SUCCESS)
            {
                *Cp = rp; *Ci = ri;
                *Cx = iso ? vx : rx;
                if (iso) vx = NULL;
            }
            else
            {
                free(rp); free(ri); free(rx);
            }
        }
    }
    free(P); free(H); free(B); free(I); free(X);
    free(vp); free(vi); free(vx);
    return rc;
}

//------------------------------------------------------------------------------
// encode: sparse, uncompressed; p/i are compressed by row, or by column when
// by_col (p then has ncols+1 entries and i holds row indices)
//------------------------------------------------------------------------------

int grb_b200_blob_encode(void *blob_out, size_t *blob_size, int64_t nrows, int64_t ncols,
                         int type, const int64_t *p, const int64_t *i, const void *x,
                         bool iso, bool by_col)
{
    if (!blob_size || !p) return S_NULL;
    const size_t ts = type_bytes(type);
    if (ts == 0) return S_DOMAIN;
    if (nrows < 0 || ncols < 0) return S_INVALID_VALUE;
    const int64_t vdim = by_col ? ncols : nrows, vlen = by_col ? nrows : ncols;
    const int64_t nnz = p[vdim];
    if (nnz > 0 && !i) return S_NULL;
    const int64_t lens[5] = {8 * (vdim + 1), 0, 0, 8 * nnz, (int64_t)ts * (iso ? 1 : nnz)};
    int32_t nb[5];
    size_t need = HEADER_SIZE;
    for (int a = 0; a < 5; a++)
    {
        nb[a] = lens[a] > 0 ? 1 : 0;
        need += 8 * (size_t)nb[a] + (size_t)lens[a];
    }
    const char *tname = type_name(type);
    need += 1 + strlen(tname) + 1;
    if (!blob_out) { *blob_size = need; return S_SUCCESS; }   // size query
    if (*blob_size < need) return S_INSUFFICIENT;
    if (lens[4] > 0 && !x) return S_NULL;
    uint8_t *blob = (uint8_t *)blob_out;
    size_t s = 0;
    #define WR(v, T) do { T t_ = (T)(v); memcpy(blob + s, &t_, sizeof(T)); s += sizeof(T); } while (0)
    int64_t nonempty = 0;
    for (int64_t v = 0; v < vdim; v++) nonempty += p[v + 1] > p[v];
    WR(need, uint64_t); WR(type, int32_t); WR(VERSION_9_3_1, int32_t);
    WR(vlen, int64_t); WR(vdim, int64_t); WR(vdim, int64_t); WR(nonempty, int64_t);
    WR(nnz, int64_t); WR(ts, int64_t);
    for (int a = 0; a < 5; a++) WR(lens[a], int64_t);
    WR(0.0625f, float); WR(0.04f, float);
    WR(HYPER + SPARSE + BITMAP + FULL, int32_t);      // sparsity control: automatic
    WR(4 * SPARSE + (iso ? 2 : 0) + (by_col ? 1 : 0), int32_t);
    for (int a = 0; a < 5; a++) { WR(nb[a], int32_t); WR(M_NONE, int32_t); }
    for (int a = 0; a < 5; a++) if (nb[a]) WR(lens[a], int64_t);
    memcpy(blob + s, p, (size_t)lens[0]); s += (size_t)lens[0];
    if (lens[3]) { memcpy(blob + s, i, (size_t)lens[3]); s += (size_t)lens[3]; }
    if (lens[4]) { memcpy(blob + s, x, (size_t)lens[4]); s += (size_t)lens[4]; }
    blob[s++] = 0;                                   // no matrix name
    memcpy(blob + s, tname, strlen(tname));
    s += strlen(tname);
    blob[s++] = 0;
    #undef WR
    *blob_size = s;
    return s == need ? S_SUCCESS : S_INVALID_OBJECT;
}
