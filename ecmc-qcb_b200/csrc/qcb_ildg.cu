// qcb_ildg.cpp -- ILDG configuration files in LIME framing, without c-lime.
//
// Replaces save_ildg_clime / read_ildg_clime (src/io/ildg.cpp:34-237).  LIME record
// layout (Lattice QCD Interchange Message Encapsulation): a 144-byte header
//     [0,4)   magic 0x456789ab, big-endian
//     [4,6)   format version 1, big-endian
//     [6]     flags: 0x80 = message begin (MB), 0x40 = message end (ME)
//     [8,16)  payload length in bytes, big-endian
//     [16,144) record type, NUL padded
// followed by the payload, zero-padded to a multiple of 8 bytes.
// The writer emits what the reference emits: an "ildg-format" XML record (MB=1, ME=1,
// ildg.cpp:13-22,59) and an "ildg-binary-data" record (MB=0, ME=1, ildg.cpp:67) holding
// big-endian FP64 links in site order t,z,y,x (x fastest), mu = x,y,z,t, row-major 3x3.
// The reader accepts 64- and 32-bit payloads and non-hypercubic extents; it rejects a
// payload whose size does not match the lattice (ildg.cpp:142-168).
//
// SciDAC checksums (the USQCD QIO site checksum; the reference neither writes nor checks them):
// for the site of lexicographic rank r (the payload's site order) with bytes b_r as stored,
// c_r = CRC-32(b_r) (the ISO-HDLC / zlib CRC: reflected polynomial 0xEDB88320, initial and final
// XOR 0xFFFFFFFF), suma = XOR_r rotl(c_r, r mod 29), sumb = XOR_r rotl(c_r, r mod 31).  They
// travel as a "scidac-checksum" record, <scidacChecksum><version>1.0</version><suma>hex</suma>
// <sumb>hex</sumb></scidacChecksum>, after the binary record.  The writer adds it on request
// only, so its default output stays byte-identical to the reference's; the reader checks it
// whenever a file carries one.
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <thread>
#include <vector>

#include "qcb_internal.h"

using namespace qcb;

namespace {

const uint32_t kLimeMagic = 0x456789abu;

void put_be32(unsigned char* p, uint32_t v) {
    for (int i = 0; i < 4; i++) p[i] = (unsigned char)(v >> (24 - 8 * i));
}
void put_be16(unsigned char* p, uint16_t v) {
    p[0] = (unsigned char)(v >> 8);
    p[1] = (unsigned char)v;
}
void put_be64(unsigned char* p, uint64_t v) {
    for (int i = 0; i < 8; i++) p[i] = (unsigned char)(v >> (56 - 8 * i));
}
uint32_t get_be32(const unsigned char* p) {
    return ((uint32_t)p[0] << 24) | ((uint32_t)p[1] << 16) | ((uint32_t)p[2] << 8) | p[3];
}
uint64_t get_be64(const unsigned char* p) {
    uint64_t v = 0;
    for (int i = 0; i < 8; i++) v = (v << 8) | p[i];
    return v;
}

bool write_header(FILE* fp, const char* type, uint64_t len, bool mb, bool me) {
    unsigned char h[144];
    memset(h, 0, sizeof(h));
    put_be32(h, kLimeMagic);
    put_be16(h + 4, 1);
    h[6] = (unsigned char)((mb ? 0x80 : 0) | (me ? 0x40 : 0));
    put_be64(h + 8, len);
    strncpy((char*)h + 16, type, 128);
    return fwrite(h, 1, 144, fp) == 144;
}

// generate_ildg_xml (src/io/ildg.cpp:13-22), extended to non-hypercubic extents.
std::string ildg_xml(const int L[4], int precision) {
    char buf[512];
    snprintf(buf, sizeof(buf),
             "<?xml version=\"1.0\" encoding=\"UTF-8\"?>\n"
             "<ildgFormat><version>1.0</version><field>su3gauge</field>"
             "<precision>%d</precision><lx>%d</lx><ly>%d</ly><lz>%d</lz><lt>%d</lt>"
             "</ildgFormat>",
             precision, L[0], L[1], L[2], L[3]);
    return std::string(buf);
}

bool xml_int(const std::string& xml, const char* tag, int* out) {
    std::string open = std::string("<") + tag + ">";
    size_t p = xml.find(open);
    if (p == std::string::npos) return false;
    p += open.size();
    size_t q = xml.find('<', p);
    if (q == std::string::npos) return false;
    std::string v = xml.substr(p, q - p);
    char* end = nullptr;
    long x = strtol(v.c_str(), &end, 10);
    if (end == v.c_str()) return false;
    *out = (int)x;
    return true;
}

// CRC-32 by slicing-by-8: T[0] is the byte-wise table of the reflected polynomial, and
// T[k][i] = (T[k-1][i] >> 8) ^ T[0][T[k-1][i] & 0xff] advances a byte's contribution by k more
// bytes, so eight input bytes fold into the register with eight lookups.
struct Crc32Tables {
    uint32_t t[8][256];
    Crc32Tables() {
        for (uint32_t i = 0; i < 256; i++) {
            uint32_t c = i;
            for (int k = 0; k < 8; k++) c = (c & 1) ? (c >> 1) ^ 0xEDB88320u : c >> 1;
            t[0][i] = c;
        }
        for (int k = 1; k < 8; k++)
            for (int i = 0; i < 256; i++) t[k][i] = (t[k - 1][i] >> 8) ^ t[0][t[k - 1][i] & 0xff];
    }
};

uint32_t crc32(const unsigned char* p, size_t n) {
    static const Crc32Tables tab;
    const auto& t = tab.t;
    uint32_t c = 0xFFFFFFFFu;
    for (; n >= 8; n -= 8, p += 8) {
        const uint32_t lo = c ^ ((uint32_t)p[0] | (uint32_t)p[1] << 8 | (uint32_t)p[2] << 16 | (uint32_t)p[3] << 24);
        c = t[7][lo & 0xff] ^ t[6][(lo >> 8) & 0xff] ^ t[5][(lo >> 16) & 0xff] ^ t[4][lo >> 24] ^ t[3][p[4]] ^
            t[2][p[5]] ^ t[1][p[6]] ^ t[0][p[7]];
    }
    for (; n > 0; n--, p++) c = t[0][(c ^ *p) & 0xff] ^ (c >> 8);
    return c ^ 0xFFFFFFFFu;
}

inline uint32_t rotl32(uint32_t v, unsigned r) { return r ? (v << r) | (v >> (32 - r)) : v; }

// SciDAC suma / sumb of n_sites records of site_bytes each; sites split over host threads (the
// XOR sums do not depend on the order).
void scidac_sums(const unsigned char* data, uint64_t n_sites, size_t site_bytes, uint32_t* suma, uint32_t* sumb) {
    const unsigned hw = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    const uint64_t per = std::max<uint64_t>(4096, (n_sites + hw - 1) / hw);
    const unsigned nt = (unsigned)std::max<uint64_t>(1, (n_sites + per - 1) / per);
    std::vector<uint32_t> a(nt, 0), b(nt, 0);
    auto work = [&](unsigned k) {
        const uint64_t r0 = k * per, r1 = std::min(n_sites, r0 + per);
        uint32_t x = 0, y = 0;
        for (uint64_t r = r0; r < r1; r++) {
            const uint32_t c = crc32(data + r * site_bytes, site_bytes);
            x ^= rotl32(c, (unsigned)(r % 29));
            y ^= rotl32(c, (unsigned)(r % 31));
        }
        a[k] = x;
        b[k] = y;
    };
    std::vector<std::thread> th;
    for (unsigned k = 1; k < nt; k++) th.emplace_back(work, k);
    work(0);
    for (auto& t : th) t.join();
    uint32_t x = 0, y = 0;
    for (unsigned k = 0; k < nt; k++) {
        x ^= a[k];
        y ^= b[k];
    }
    *suma = x;
    *sumb = y;
}

std::string scidac_xml(uint32_t suma, uint32_t sumb) {
    char buf[256];
    snprintf(buf, sizeof(buf),
             "<?xml version=\"1.0\" encoding=\"UTF-8\"?><scidacChecksum><version>1.0</version>"
             "<suma>%x</suma><sumb>%x</sumb></scidacChecksum>",
             suma, sumb);
    return buf;
}

// Hex value of <tag>...</tag>; false when absent or not hexadecimal.
bool xml_hex(const std::string& xml, const char* tag, uint32_t* v) {
    const std::string open = std::string("<") + tag + ">";
    size_t a = xml.find(open);
    if (a == std::string::npos) return false;
    a += open.size();
    while (a < xml.size() && isspace((unsigned char)xml[a])) a++;
    char* end = nullptr;
    const unsigned long x = strtoul(xml.c_str() + a, &end, 16);
    if (end == xml.c_str() + a || x > 0xFFFFFFFFul) return false;
    *v = (uint32_t)x;
    return true;
}

struct LimeScan {
    bool have_xml = false;
    int L[4] = {0, 0, 0, 0};
    int precision = 0;
    bool have_bin = false;
    long bin_offset = 0;
    uint64_t bin_len = 0;
    bool have_sum = false;
    uint32_t suma = 0, sumb = 0;
};

// Walks the LIME records of the file, reading the "ildg-format" XML and locating the
// "ildg-binary-data" payload (read_ildg_clime's record loop, ildg.cpp:155-175).
int scan(FILE* fp, LimeScan* s) {
    unsigned char h[144];
    long pos = 0;
    int nrec = 0;
    while (true) {
        if (fseek(fp, pos, SEEK_SET) != 0) return fail(QCB_EIO, "seek failed");
        size_t n = fread(h, 1, 144, fp);
        if (n == 0) break;
        if (n != 144) return fail(QCB_EFORMAT, "truncated LIME header at offset %ld", pos);
        if (get_be32(h) != kLimeMagic) return fail(QCB_EFORMAT, "bad LIME magic at offset %ld", pos);
        uint64_t len = get_be64(h + 8);
        char type[129];
        memcpy(type, h + 16, 128);
        type[128] = 0;
        long data = pos + 144;
        if (strcmp(type, "ildg-format") == 0 && len < (1u << 20)) {
            std::string xml((size_t)len, '\0');
            if (fread(&xml[0], 1, (size_t)len, fp) != len) return fail(QCB_EFORMAT, "truncated ildg-format record");
            int ok = 1;
            ok &= xml_int(xml, "lx", &s->L[0]);
            ok &= xml_int(xml, "ly", &s->L[1]);
            ok &= xml_int(xml, "lz", &s->L[2]);
            ok &= xml_int(xml, "lt", &s->L[3]);
            if (!xml_int(xml, "precision", &s->precision)) s->precision = 0;
            s->have_xml = ok != 0;
        } else if (strcmp(type, "scidac-checksum") == 0 && len < (1u << 16) && !s->have_sum) {
            std::string xml((size_t)len, '\0');
            if (fread(&xml[0], 1, (size_t)len, fp) != len) return fail(QCB_EFORMAT, "truncated scidac-checksum record");
            if (!xml_hex(xml, "suma", &s->suma) || !xml_hex(xml, "sumb", &s->sumb))
                return fail(QCB_EFORMAT, "scidac-checksum record without hexadecimal suma/sumb");
            s->have_sum = true;
        } else if (strcmp(type, "ildg-binary-data") == 0 && !s->have_bin) {
            s->have_bin = true;
            s->bin_offset = data;
            s->bin_len = len;
        }
        nrec++;
        uint64_t padded = (len + 7) & ~(uint64_t)7;
        pos = data + (long)padded;
    }
    if (nrec == 0) return fail(QCB_EFORMAT, "empty file");
    return QCB_OK;
}

}  // namespace

extern "C" {

int qcb_scidac_checksum(const void* payload, uint64_t n_sites, uint64_t site_bytes, uint32_t* suma, uint32_t* sumb) {
    if ((!payload && n_sites > 0) || !suma || !sumb || site_bytes == 0) return fail(QCB_EINVAL, "null argument");
    scidac_sums((const unsigned char*)payload, n_sites, (size_t)site_bytes, suma, sumb);
    return QCB_OK;
}

int qcb_ildg_write(qcb_field f, const char* path) { return qcb_ildg_write_ex(f, path, 0); }

int qcb_ildg_write_ex(qcb_field f, const char* path, int flags) {
    if (!f || !path) return fail(QCB_EINVAL, "null argument");
    if (flags & ~QCB_ILDG_SCIDAC_CHECKSUM) return fail(QCB_EINVAL, "unknown ILDG write flags 0x%x", flags);
    const bool with_sum = (flags & QCB_ILDG_SCIDAC_CHECKSUM) != 0;
    const size_t nd = (size_t)f->g.V * 72;
    std::vector<double> buf(nd);
    int r = field_download_host(f, buf.data(), 1);
    if (r != QCB_OK) return r;
    FILE* fp = fopen(path, "wb");
    if (!fp) return fail(QCB_EIO, "cannot open %s for writing", path);
    std::string xml = ildg_xml(f->L, 64);
    bool ok = write_header(fp, "ildg-format", xml.size(), true, true);
    ok = ok && fwrite(xml.data(), 1, xml.size(), fp) == xml.size();
    static const char zeros[8] = {0};
    size_t pad = (8 - xml.size() % 8) % 8;
    ok = ok && fwrite(zeros, 1, pad, fp) == pad;
    // with a checksum the binary record no longer ends the message: the checksum record does
    ok = ok && write_header(fp, "ildg-binary-data", (uint64_t)nd * 8, false, !with_sum);
    ok = ok && fwrite(buf.data(), 8, nd, fp) == nd;
    if (with_sum) {
        uint32_t a = 0, b = 0;
        scidac_sums((const unsigned char*)buf.data(), (uint64_t)f->g.V, 72 * 8, &a, &b);
        const std::string sx = scidac_xml(a, b);
        ok = ok && write_header(fp, "scidac-checksum", sx.size(), false, true);
        ok = ok && fwrite(sx.data(), 1, sx.size(), fp) == sx.size();
        const size_t spad = (8 - sx.size() % 8) % 8;
        ok = ok && fwrite(zeros, 1, spad, fp) == spad;
    }
    ok = (fclose(fp) == 0) && ok;
    if (!ok) return fail(QCB_EIO, "write failed: %s", path);
    return QCB_OK;
}

int qcb_ildg_probe(const char* path, int L[4], int* precision) {
    if (!path) return fail(QCB_EINVAL, "null path");
    FILE* fp = fopen(path, "rb");
    if (!fp) return fail(QCB_EIO, "cannot open %s", path);
    LimeScan s;
    int r = scan(fp, &s);
    fclose(fp);
    if (r != QCB_OK) return r;
    if (!s.have_xml) return fail(QCB_EFORMAT, "no ildg-format record in %s", path);
    if (L)
        for (int d = 0; d < 4; d++) L[d] = s.L[d];
    if (precision) *precision = s.precision;
    return QCB_OK;
}

int qcb_ildg_read(qcb_field f, const char* path) {
    if (!f || !path) return fail(QCB_EINVAL, "null argument");
    FILE* fp = fopen(path, "rb");
    if (!fp) return fail(QCB_EIO, "cannot open %s", path);
    LimeScan s;
    int r = scan(fp, &s);
    if (r != QCB_OK) {
        fclose(fp);
        return r;
    }
    if (!s.have_bin) {
        fclose(fp);
        return fail(QCB_EFORMAT, "record 'ildg-binary-data' not found in %s", path);
    }
    if (s.have_xml)
        for (int d = 0; d < 4; d++)
            if (s.L[d] != f->L[d]) {
                fclose(fp);
                return fail(QCB_EFORMAT, "lattice %dx%dx%dx%d in file, %dx%dx%dx%d in field", s.L[0], s.L[1], s.L[2],
                            s.L[3], f->L[0], f->L[1], f->L[2], f->L[3]);
            }
    const uint64_t n = (uint64_t)f->g.V * 72;
    int prec = s.precision;
    if (prec != 32 && prec != 64) prec = (s.bin_len == n * 4) ? 32 : 64;
    if (s.bin_len != n * (uint64_t)(prec / 8)) {
        fclose(fp);
        return fail(QCB_EFORMAT, "binary size %llu does not match %llu links at %d bits", (unsigned long long)s.bin_len,
                    (unsigned long long)(n / 18), prec);
    }
    std::vector<double> buf(n);
    bool ok = fseek(fp, s.bin_offset, SEEK_SET) == 0;
    uint32_t a = 0, b = 0;
    if (ok && prec == 64) {
        ok = fread(buf.data(), 8, n, fp) == n;
        if (ok && s.have_sum) scidac_sums((const unsigned char*)buf.data(), (uint64_t)f->g.V, 72 * 8, &a, &b);
    } else if (ok) {
        std::vector<uint32_t> b32(n);
        ok = fread(b32.data(), 4, n, fp) == n;
        if (ok && s.have_sum) scidac_sums((const unsigned char*)b32.data(), (uint64_t)f->g.V, 72 * 4, &a, &b);
        for (uint64_t i = 0; ok && i < n; i++) {
            uint32_t v = __builtin_bswap32(b32[i]);
            float x;
            memcpy(&x, &v, 4);
            buf[i] = (double)x;
        }
    }
    fclose(fp);
    if (!ok) return fail(QCB_EFORMAT, "truncated binary payload in %s", path);
    if (s.have_sum && (a != s.suma || b != s.sumb))
        return fail(QCB_EFORMAT, "SciDAC checksum mismatch in %s: file %x %x, payload %x %x", path, s.suma, s.sumb, a, b);
    return field_upload_host(f, buf.data(), prec == 64 ? 1 : 0);
}

}  // extern "C"
