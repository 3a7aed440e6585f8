// Blosc2 contiguous-frame reader/writer and the chunk header helpers used on the host.
//
// Replaces, for containers of this library, blosc2_schunk_copy / blosc2_schunk_open /
// blosc2_schunk_to_buffer as called by iarray_container_save / _load / _open and
// iarray_to_cframe / iarray_from_cframe (src/iarray_container.c:50-300).  The byte
// layout (msgpack header with the "caterva" and "iarray" metalayers, chunks back to
// back, a memcpyed offsets chunk, msgpack trailer) is the one of the reference's own
// frames tests/data/test_<distribution>.iarray; the "iarray" metalayer follows
// _iarray_serialize_meta (src/iarray_private.h:364-387).
#include "frame.h"

#include <string.h>

namespace iab {

static void put_be(std::vector<uint8_t> &v, uint64_t x, int nbytes)
{
    for (int i = nbytes - 1; i >= 0; i--) v.push_back((uint8_t)(x >> (8 * i)));
}
static uint64_t get_be(const uint8_t *p, int nbytes)
{
    uint64_t x = 0;
    for (int i = 0; i < nbytes; i++) x = (x << 8) | p[i];
    return x;
}
static int32_t rd_le32(const uint8_t *p) { int32_t v; memcpy(&v, p, 4); return v; }

std::vector<uint8_t> caterva_meta(int ndim, const int64_t *shape, const int64_t *chunk, const int64_t *block)
{
    std::vector<uint8_t> m;
    m.push_back(0x95);
    m.push_back(0);                 // version
    m.push_back((uint8_t)ndim);
    m.push_back((uint8_t)(0x90 + ndim));
    for (int i = 0; i < ndim; i++) { m.push_back(0xd3); put_be(m, (uint64_t)shape[i], 8); }
    m.push_back((uint8_t)(0x90 + ndim));
    for (int i = 0; i < ndim; i++) { m.push_back(0xd2); put_be(m, (uint32_t)chunk[i], 4); }
    m.push_back((uint8_t)(0x90 + ndim));
    for (int i = 0; i < ndim; i++) { m.push_back(0xd2); put_be(m, (uint32_t)block[i], 4); }
    return m;
}

std::vector<uint8_t> iarray_meta(int dtype)
{
    return {0x93, 0x00, (uint8_t)dtype, 0x00};
}

std::vector<uint8_t> memcpyed_chunk(const uint8_t *data, int32_t nbytes, int typesize)
{
    std::vector<uint8_t> c(32 + (size_t)nbytes, 0);
    c[0] = 5; c[1] = 1; c[2] = 0x07; c[3] = (uint8_t)typesize;
    int32_t cb = nbytes + 32;
    memcpy(&c[4], &nbytes, 4);
    memcpy(&c[8], &nbytes, 4);
    memcpy(&c[12], &cb, 4);
    c[16 + 5] = 1;
    if (nbytes) memcpy(&c[32], data, nbytes);
    return c;
}

static const uint8_t kTrailer[35] = {0x94, 0x01, 0x93, 0xcd, 0x00, 0x06, 0xde, 0x00, 0x00, 0xdc, 0x00, 0x00,
                                     0xce, 0x00, 0x00, 0x00, 0x23, 0xd8, 0x00};

std::vector<uint8_t> frame_tail(const std::vector<int32_t> &lens, bool sparse)
{
    std::vector<int64_t> offsets;
    int64_t acc = 0;
    for (int32_t l : lens) { offsets.push_back(sparse ? (int64_t)offsets.size() : acc); acc += l; }
    std::vector<uint8_t> t = memcpyed_chunk(reinterpret_cast<const uint8_t *>(offsets.data()),
                                            (int32_t)(offsets.size() * 8), 8);
    // trailer: [version, [vlmeta index size, {}, []], trailer length, fingerprint]
    t.insert(t.end(), kTrailer, kTrailer + 35);
    return t;
}

std::vector<uint8_t> frame_header(const FrameInfo &fi, int64_t data_cbytes, int64_t nchunks)
{
    std::vector<uint8_t> h;
    const std::vector<uint8_t> cat = caterva_meta(fi.ndim, fi.shape, fi.chunk, fi.block);
    const std::vector<uint8_t> ia = iarray_meta(fi.dtype);
    h.push_back(0x9e);
    h.push_back(0xa8);
    const char magic[8] = {'b', '2', 'f', 'r', 'a', 'm', 'e', 0};
    h.insert(h.end(), magic, magic + 8);
    h.push_back(0xd2); put_be(h, 0, 4);                 // header size, patched below
    h.push_back(0xcf); put_be(h, 0, 8);                 // frame size, patched below
    h.push_back(0xa4);
    h.push_back(0x12);                                  // frame format 2, 64-bit offsets
    h.push_back(fi.sparse ? 0x01 : 0x00);               // frame type: contiguous / directory
    h.push_back((uint8_t)((fi.clevel << 4) | (fi.codec & 0x0f)));
    h.push_back(0x00);
    h.push_back(0xd3); put_be(h, (uint64_t)fi.nbytes, 8);
    h.push_back(0xd3); put_be(h, (uint64_t)data_cbytes, 8);
    h.push_back(0xd2); put_be(h, (uint32_t)fi.typesize, 4);
    h.push_back(0xd2); put_be(h, (uint32_t)fi.blocksize, 4);
    h.push_back(0xd2); put_be(h, (uint32_t)fi.chunksize, 4);
    h.push_back(0xd1); put_be(h, (uint16_t)fi.nthreads, 2);
    h.push_back(0xd1); put_be(h, (uint16_t)fi.nthreads, 2);
    h.push_back(0xc2);                                  // no user metalayers
    h.push_back(0xd8); h.push_back(0x06);               // filter pipeline (fixext 16)
    for (int i = 0; i < 6; i++) h.push_back(i == 5 ? (uint8_t)(fi.shuffle ? 1 : 0) : 0);
    h.push_back((uint8_t)fi.codec);
    h.push_back(0);
    for (int i = 0; i < 8; i++) h.push_back(0);
    // metalayers: [index map size, {name: offset}, [contents]]
    const size_t idx_pos = h.size();
    h.push_back(0x93);
    h.push_back(0xcd); put_be(h, 0, 2);
    h.push_back(0xde); put_be(h, 2, 2);
    const char *names[2] = {"caterva", "iarray"};
    size_t off_pos[2];
    for (int i = 0; i < 2; i++) {
        const size_t nl = strlen(names[i]);
        h.push_back((uint8_t)(0xa0 + nl));
        h.insert(h.end(), names[i], names[i] + nl);
        h.push_back(0xd2);
        off_pos[i] = h.size();
        put_be(h, 0, 4);
    }
    const uint16_t map_size = (uint16_t)(h.size() - idx_pos);
    h[idx_pos + 2] = (uint8_t)(map_size >> 8);
    h[idx_pos + 3] = (uint8_t)map_size;
    h.push_back(0xdc); put_be(h, 2, 2);
    const std::vector<uint8_t> *contents[2] = {&cat, &ia};
    for (int i = 0; i < 2; i++) {
        const uint32_t pos = (uint32_t)h.size();
        for (int k = 0; k < 4; k++) h[off_pos[i] + k] = (uint8_t)(pos >> (8 * (3 - k)));
        h.push_back(0xc6); put_be(h, (uint32_t)contents[i]->size(), 4);
        h.insert(h.end(), contents[i]->begin(), contents[i]->end());
    }
    const uint32_t header_size = (uint32_t)h.size();
    for (int k = 0; k < 4; k++) h[11 + k] = (uint8_t)(header_size >> (8 * (3 - k)));
    // a sparse frame's index file holds no chunk bytes
    const uint64_t fs = (uint64_t)h.size() + (fi.sparse ? 0 : (uint64_t)data_cbytes) + 32 + 8 * (uint64_t)nchunks + 35;
    for (int k = 0; k < 8; k++) h[16 + k] = (uint8_t)(fs >> (8 * (7 - k)));
    return h;
}

bool write_frame(const FrameInfo &fi, const std::vector<const uint8_t *> &chunks, const std::vector<int32_t> &lens,
                 std::vector<uint8_t> *out)
{
    int64_t data_cbytes = 0;
    for (int32_t l : lens) data_cbytes += l;
    *out = frame_header(fi, data_cbytes, (int64_t)lens.size());
    for (size_t i = 0; i < chunks.size(); i++) out->insert(out->end(), chunks[i], chunks[i] + lens[i]);
    const std::vector<uint8_t> t = frame_tail(lens);
    out->insert(out->end(), t.begin(), t.end());
    return true;
}

// Minimal msgpack integer reader for the fixed header fields.
static bool mp_int(const uint8_t *b, size_t n, size_t &p, int64_t *v)
{
    if (p >= n) return false;
    const uint8_t t = b[p];
    if (t < 0x80) { *v = t; p += 1; return true; }
    int sz;
    bool sgn;
    switch (t) {
    case 0xcc: sz = 1; sgn = false; break;
    case 0xcd: sz = 2; sgn = false; break;
    case 0xce: sz = 4; sgn = false; break;
    case 0xcf: sz = 8; sgn = false; break;
    case 0xd0: sz = 1; sgn = true; break;
    case 0xd1: sz = 2; sgn = true; break;
    case 0xd2: sz = 4; sgn = true; break;
    case 0xd3: sz = 8; sgn = true; break;
    default: return false;
    }
    if (p + 1 + sz > n) return false;
    uint64_t u = get_be(b + p + 1, sz);
    if (sgn && sz < 8 && (u >> (8 * sz - 1))) u |= ~0ull << (8 * sz);
    *v = (int64_t)u;
    p += 1 + sz;
    return true;
}

bool read_frame(const uint8_t *b, size_t n, FrameInfo *fi, std::vector<std::pair<int64_t, int32_t>> *chunks,
                std::string *why)
{
    auto fail = [&](const char *m) { if (why) *why = m; return false; };
    if (n < 90 || b[0] != 0x9e || b[1] != 0xa8 || memcmp(b + 2, "b2frame", 8) != 0) return fail("not a blosc2 frame");
    size_t p = 10;
    int64_t header_size, frame_size, v;
    if (!mp_int(b, n, p, &header_size)) return fail("header size");
    if (!mp_int(b, n, p, &frame_size)) return fail("frame size");
    if (frame_size > (int64_t)n || header_size > frame_size) return fail("truncated frame");
    if (b[p] != 0xa4) return fail("flags");
    if (b[p + 2] > 1) return fail("frame type");
    fi->sparse = b[p + 2] == 1;
    fi->codec = b[p + 3] & 0x0f;
    fi->clevel = b[p + 3] >> 4;
    p += 5;
    if (!mp_int(b, n, p, &fi->nbytes)) return fail("nbytes");
    if (!mp_int(b, n, p, &v)) return fail("cbytes");
    if (!mp_int(b, n, p, &v)) return fail("typesize");
    fi->typesize = (int)v;
    if (!mp_int(b, n, p, &v)) return fail("blocksize");
    fi->blocksize = (int32_t)v;
    if (!mp_int(b, n, p, &v)) return fail("chunksize");
    fi->chunksize = (int32_t)v;
    if (!mp_int(b, n, p, &v)) return fail("nthreads");
    fi->nthreads = (int)v;
    if (!mp_int(b, n, p, &v)) return fail("nthreads");
    if (b[p] != 0xc2 && b[p] != 0xc3) return fail("usermeta flag");
    p += 1;
    if (b[p] != 0xd8) return fail("filter pipeline");
    fi->shuffle = b[p + 2 + 5] == 1;
    p += 18;
    if (b[p] != 0x93) return fail("metalayers");
    p += 1;
    if (!mp_int(b, n, p, &v)) return fail("metalayer index");
    if (b[p] != 0xde) return fail("metalayer map");
    const int nmeta = (int)get_be(b + p + 1, 2);
    p += 3;
    std::vector<std::string> names;
    for (int i = 0; i < nmeta; i++) {
        if (p >= n || (b[p] & 0xe0) != 0xa0) return fail("metalayer name");
        const int nl = b[p] & 0x1f;
        names.emplace_back((const char *)b + p + 1, nl);
        p += 1 + nl;
        if (!mp_int(b, n, p, &v)) return fail("metalayer offset");
    }
    if (b[p] != 0xdc) return fail("metalayer contents");
    p += 3;
    bool have_cat = false, have_ia = false;
    for (int i = 0; i < nmeta; i++) {
        if (b[p] != 0xc6) return fail("metalayer bin");
        const uint32_t ln = (uint32_t)get_be(b + p + 1, 4);
        const uint8_t *m = b + p + 5;
        if (p + 5 + ln > (size_t)header_size) return fail("metalayer size");
        if (names[i] == "caterva") {
            if (ln < 3 || m[0] != 0x95) return fail("caterva meta");
            fi->ndim = m[2];
            if (fi->ndim < 1 || fi->ndim > 8) return fail("caterva ndim");
            size_t q = 3;
            int64_t *dst[3] = {fi->shape, fi->chunk, fi->block};
            for (int a = 0; a < 3; a++) {
                if (m[q] != 0x90 + fi->ndim) return fail("caterva array");
                q += 1;
                for (int d = 0; d < fi->ndim; d++) {
                    int64_t x;
                    if (!mp_int(m, ln, q, &x)) return fail("caterva value");
                    dst[a][d] = x;
                }
            }
            have_cat = true;
        } else if (names[i] == "iarray") {
            if (ln < 3 || m[0] != 0x93) return fail("iarray meta");
            fi->dtype = m[2];
            have_ia = true;
        }
        p += 5 + ln;
    }
    if (!have_cat) return fail("missing caterva metalayer");
    if (!have_ia) fi->dtype = fi->typesize == 8 ? 0 : 1;
    const int64_t nchunks = fi->chunksize > 0 ? (fi->nbytes + fi->chunksize - 1) / fi->chunksize : 0;
    size_t pos = (size_t)header_size;
    for (int64_t c = 0; c < nchunks && !fi->sparse; c++) {
        if (pos + 32 > n) return fail("chunk past end");
        pos += (size_t)rd_le32(b + pos + 12);
    }
    if (pos + 32 > n) return fail("offsets chunk missing");
    const uint8_t *oc = b + pos;
    const int32_t onb = rd_le32(oc + 4), ocb = rd_le32(oc + 12);
    if (!(oc[2] & 0x02) || ocb < 32 + onb || onb != nchunks * 8) return fail("offsets chunk is not memcpyed");
    chunks->clear();
    for (int64_t c = 0; c < nchunks; c++) {
        int64_t off;
        memcpy(&off, oc + 32 + 8 * c, 8);
        if (fi->sparse) {
            if (off < 0 || off > 0xFFFFFFFFll) return fail("chunk file number out of range");
            chunks->emplace_back(off, 0);
            continue;
        }
        const size_t s = (size_t)header_size + (size_t)off;
        if (s + 32 > n) return fail("chunk offset out of range");
        const int32_t cb = rd_le32(b + s + 12);
        if (cb < 32 || s + (size_t)cb > n) return fail("chunk size out of range");
        chunks->emplace_back((int64_t)s, cb);
    }
    return true;
}

}  // namespace iab
