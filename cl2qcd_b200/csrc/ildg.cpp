// ildg.cpp -- reader for gauge configurations in ILDG format inside LIME files
// (the reference reads them in ildg_io/ildgIo_gaugefield.cpp through the LIME
// library; this is a self-contained reader of the published formats).
//
// LIME: a sequence of records, each a 144-byte big-endian header (magic
// 0x456789ab, version, flags, payload length in bytes, 128-byte type string)
// followed by the payload padded to a multiple of 8 bytes.  ILDG: the record
// "ildg-format" holds XML with <precision> (32 or 64) and <lx> <ly> <lz> <lt>;
// "ildg-binary-data" holds the links as big-endian IEEE numbers, site by site
// with x fastest (then y, z, t), per site the four directions x, y, z, t, per
// link the 3x3 complex matrix row by row; "scidac-checksum" holds the SciDAC
// checksum <suma>, <sumb> (hex): for the site of rank r (its position in the
// file), c = CRC-32 of its bytes, suma ^= rotl(c, r mod 29), sumb ^= rotl(c, r mod 31).
//
// The reader returns the reference's host layout Matrixsu3[4V] with link
// mu + 4*site (site = x + NS y + NS^2 z + NS^3 t, mu = 0 the time direction):
// ILDG direction l (0 = x ... 3 = t) becomes mu = (l + 1) mod 4, as the
// reference stores it (ildgIo_gaugefield.cpp, copy_gaugefield_from_ildg_format).
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/cl2qcd_b200.h"

namespace {

uint64_t be64(const unsigned char* p)
{
    uint64_t v = 0;
    for (int i = 0; i < 8; ++i) v = (v << 8) | p[i];
    return v;
}
uint32_t be32(const unsigned char* p) { return (uint32_t)p[0] << 24 | (uint32_t)p[1] << 16 | (uint32_t)p[2] << 8 | p[3]; }

// CRC-32 (IEEE 802.3, reflected polynomial 0xEDB88320), table-driven
struct Crc32 {
    uint32_t t[256];
    Crc32()
    {
        for (uint32_t i = 0; i < 256; ++i) {
            uint32_t c = i;
            for (int k = 0; k < 8; ++k) c = (c & 1) ? 0xEDB88320u ^ (c >> 1) : c >> 1;
            t[i] = c;
        }
    }
    uint32_t operator()(const unsigned char* p, size_t n) const
    {
        uint32_t c = 0xFFFFFFFFu;
        for (size_t i = 0; i < n; ++i) c = t[(c ^ p[i]) & 0xFF] ^ (c >> 8);
        return c ^ 0xFFFFFFFFu;
    }
};

uint32_t rotl(uint32_t x, uint32_t r) { return r ? (x << r) | (x >> (32 - r)) : x; }

// the integer between <tag> and </tag>, or -1
long xml_int(const std::string& xml, const char* tag, int base = 10)
{
    const std::string open = std::string("<") + tag + ">";
    const size_t a         = xml.find(open);
    if (a == std::string::npos) return -1;
    return strtol(xml.c_str() + a + open.size(), nullptr, base);
}

}  // namespace

extern "C" {

// Reads an ILDG gauge configuration.  With aos == NULL only the header is read
// (extents, precision).  aos must hold 4 * NS^3 * NT * 18 doubles.  info (may
// be NULL) receives the "xlf-info" text, truncated to info_len.  checksum_status:
// 1 the recorded SciDAC checksum matches the data, 0 it does not, -1 none recorded;
// suma / sumb (may be NULL) receive the checksum computed from the data.
C2Q_EXPORT int c2q_ildg_read(const char* path, double* aos, size_t aos_len, int* ns, int* nt, int* precision,
                             char* info, int info_len, unsigned* suma, unsigned* sumb, int* checksum_status)
{
    if (!path || !ns || !nt || !precision) return C2Q_BAD_ARG;
    FILE* f = fopen(path, "rb");
    if (!f) return C2Q_BAD_ARG;
    std::vector<unsigned char> file;
    unsigned char buf[1 << 16];
    size_t got;
    while ((got = fread(buf, 1, sizeof buf, f)) > 0) file.insert(file.end(), buf, buf + got);
    fclose(f);

    std::string format, xlf;
    const unsigned char* data = nullptr;
    uint64_t data_len         = 0;
    long rec_a = -1, rec_b = -1;
    size_t off = 0;
    while (off + 144 <= file.size()) {
        const unsigned char* h = file.data() + off;
        if (be32(h) != 0x456789abu) return C2Q_BAD_ARG;  // not a LIME record
        const uint64_t len = be64(h + 8);
        char type[129];
        memcpy(type, h + 16, 128);
        type[128] = 0;
        // truncated record (off + 144 <= size holds; compared this way a length
        // read from a damaged header cannot wrap around), or a length whose
        // 8-byte padding would not fit a size_t
        if (len > file.size() - off - 144 || len > SIZE_MAX - 7) return C2Q_BAD_ARG;
        const unsigned char* payload = h + 144;
        const std::string t(type);
        if (t == "ildg-format") format.assign(reinterpret_cast<const char*>(payload), len);
        if (t == "xlf-info") xlf.assign(reinterpret_cast<const char*>(payload), len);
        if (t == "ildg-binary-data") {
            data     = payload;
            data_len = len;
        }
        if (t == "scidac-checksum") {
            const std::string x(reinterpret_cast<const char*>(payload), len);
            rec_a = xml_int(x, "suma", 16);
            rec_b = xml_int(x, "sumb", 16);
        }
        off += 144 + ((len + 7) / 8) * 8;
    }
    const long lx = xml_int(format, "lx"), ly = xml_int(format, "ly"), lz = xml_int(format, "lz"),
               lt = xml_int(format, "lt"), prec = xml_int(format, "precision");
    if (lx < 1 || lx != ly || lx != lz || lt < 1 || (prec != 32 && prec != 64) || !data) return C2Q_BAD_ARG;
    *ns        = (int)lx;
    *nt        = (int)lt;
    *precision = (int)prec;
    if (info && info_len > 0) {
        const size_t n = xlf.size() < (size_t)info_len - 1 ? xlf.size() : (size_t)info_len - 1;
        memcpy(info, xlf.data(), n);
        info[n] = 0;
    }
    const size_t vol       = (size_t)lx * lx * lx * lt;
    const size_t wbytes    = (size_t)prec / 8;
    const size_t site_size = 4 * 18 * wbytes;
    if (data_len != vol * site_size) return C2Q_BAD_ARG;
    // SciDAC checksum of the data as stored
    static const Crc32 crc;
    uint32_t a = 0, b = 0;
    for (size_t r = 0; r < vol; ++r) {
        const uint32_t c = crc(data + r * site_size, site_size);
        a ^= rotl(c, (uint32_t)(r % 29));
        b ^= rotl(c, (uint32_t)(r % 31));
    }
    if (suma) *suma = a;
    if (sumb) *sumb = b;
    if (checksum_status) *checksum_status = rec_a < 0 ? -1 : ((uint32_t)rec_a == a && (uint32_t)rec_b == b);
    if (!aos) return C2Q_OK;
    if (aos_len < vol * 4 * 18) return C2Q_BAD_ARG;
    for (size_t site = 0; site < vol; ++site) {
        for (int l = 0; l < 4; ++l) {
            const int mu            = (l + 1) % 4;
            double* dst             = aos + (mu + 4 * site) * 18;
            const unsigned char* src = data + site * site_size + (size_t)l * 18 * wbytes;
            for (int k = 0; k < 18; ++k) {
                const unsigned char* p = src + k * wbytes;
                if (prec == 64) {
                    const uint64_t u = be64(p);
                    double v;
                    memcpy(&v, &u, 8);
                    dst[k] = v;
                } else {
                    const uint32_t u = be32(p);
                    float v;
                    memcpy(&v, &u, 4);
                    dst[k] = v;
                }
            }
        }
    }
    return C2Q_OK;
}

}  // extern "C"
