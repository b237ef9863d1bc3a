// Wavelet coefficient files: the S2DW FITS and Matlab formats
// (src/mod/s2dw_fileio_mod.f90), written and read on the host, so that
// coefficients computed on the GPU go to and come from the files the
// reference's programs write and read (s2dw_analysis.f90:133-138,
// s2dw_synthesis, s2dw_fits2mat.f90:41-45, s2dw_maskapply.f90:69-130).
//
// FITS (fileio:796-1253): an empty primary HDU whose header carries the
// integer keywords J, B, N, BLSCOEFF and the real keyword ALPHA; image
// extensions SCOEFF_REAL and SCOEFF_IMAG (bl_scoeff x bl_scoeff); then one
// image extension WAV per scale j = 0..J holding the (2bl-1) x 2bl x N cube
// of that scale, first axis fastest; BITPIX -64 throughout.  Written here
// without CFITSIO, to the FITS standard (version 4.0): 2880-byte blocks,
// 80-character header cards, big-endian IEEE doubles.  The reader accepts
// any BITPIX and BSCALE/BZERO, as CFITSIO's ftg2dd/ftg3dd conversions do.
//
// Matlab (fileio:102-763): a .m function file with a 19-line header, the
// five parameters, a blank line, a comment line and three size lines per
// scale, then MATLAB code that loads <base>_scoeff.dat (the lower triangle
// of scoeff, real parts then imaginary parts) and <base>_wcoeff.dat (every
// scale's cube, first axis fastest), one Fortran E27.20 number per line.
// The reference's reader skips the header by line count, so the line
// structure is kept; the header's prose and the MATLAB code are this
// library's own.
#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "s2dw_internal.h"

namespace s2dw {
namespace {

constexpr int BLOCK = 2880;
constexpr int CARD = 80;

struct FileCloser {
    void operator()(FILE *f) const
    {
        if (f) fclose(f);
    }
};
using File = std::unique_ptr<FILE, FileCloser>;

// Per-scale cube sizes (2bl-1, 2bl, N) of the band limits of (J, B, alpha).
std::vector<int> scale_bl(int J, int B, double alpha)
{
    std::vector<int> bl(J + 1);
    for (int j = 0; j <= J; j++) {
        int hi = 0, lo = 0;
        band_limits(j, B, alpha, &hi, &lo);
        bl[j] = hi;
    }
    return bl;
}

int check_sizes(const char *who, int J, int B, int N, int bl_scoeff, double alpha)
{
    if (J < 0 || B < 2 || N < 1 || bl_scoeff < 0 || bl_scoeff > B || !(alpha > 1.0))
        return set_error(S2DWC_ERROR_ARG_INVALID, "%s: J=%d B=%d N=%d bl_scoeff=%d alpha=%g", who, J, B, N, bl_scoeff,
                         alpha);
    return S2DWC_OK;
}

// ---------------------------------------------------------------------------
// FITS writing
// ---------------------------------------------------------------------------
std::string pad(std::string s, size_t n)
{
    if (s.size() > n) s.resize(n);
    s.append(n - s.size(), ' ');
    return s;
}

// "KEYWORD = value / comment" with a fixed-format value (right-justified to
// column 30) or a string value (quoted, from column 11, at least 8 characters).
std::string card(const std::string &key, const std::string &value, const std::string &comment, bool is_string = false)
{
    std::string c = pad(key, 8) + "= ";
    if (is_string) {
        std::string q;
        for (char ch : value) {
            q += ch;
            if (ch == '\'') q += '\'';
        }
        c += "'" + pad(q, std::max<size_t>(8, q.size())) + "'";
    } else {
        c += std::string(value.size() < 20 ? 20 - value.size() : 0, ' ') + value;
    }
    if (!comment.empty()) c += " / " + comment;
    return pad(c, CARD);
}

std::string card_int(const std::string &key, long long v, const std::string &comment)
{
    return card(key, std::to_string(v), comment);
}

// COMMENT cards: 72 characters of text per card.
void comment_cards(std::vector<std::string> &h, const std::string &text)
{
    size_t i = 0;
    do {
        h.push_back(pad("COMMENT " + text.substr(i, 72), CARD));
        i += 72;
    } while (i < text.size());
}

int write_header(FILE *f, std::vector<std::string> h, const char *fn)
{
    h.push_back(pad("END", CARD));
    std::string blk;
    for (auto &c : h) blk += c;
    blk.append((BLOCK - blk.size() % BLOCK) % BLOCK, ' ');
    if (fwrite(blk.data(), 1, blk.size(), f) != blk.size())
        return set_error(S2DWC_ERROR_FILEIO, "writing %s: %s", fn, strerror(errno));
    return S2DWC_OK;
}

// n doubles as big-endian IEEE, element i at src[i * stride], padded with
// zeros to a whole block.
int write_doubles(FILE *f, const double *src, long long n, long long stride, const char *fn)
{
    std::vector<unsigned char> buf(1 << 20);
    long long done = 0;
    while (done < n) {
        const long long k = std::min<long long>(n - done, (long long)buf.size() / 8);
        for (long long i = 0; i < k; i++) {
            uint64_t u;
            std::memcpy(&u, src + (done + i) * stride, 8);
            for (int b = 0; b < 8; b++) buf[8 * i + b] = (unsigned char)(u >> (56 - 8 * b));
        }
        if (fwrite(buf.data(), 1, (size_t)(8 * k), f) != (size_t)(8 * k))
            return set_error(S2DWC_ERROR_FILEIO, "writing %s: %s", fn, strerror(errno));
        done += k;
    }
    const long long rem = (BLOCK - (8 * n) % BLOCK) % BLOCK;
    if (rem) {
        std::vector<unsigned char> z((size_t)rem, 0);
        if (fwrite(z.data(), 1, z.size(), f) != z.size())
            return set_error(S2DWC_ERROR_FILEIO, "writing %s: %s", fn, strerror(errno));
    }
    return S2DWC_OK;
}

std::vector<std::string> image_header(const std::vector<long long> &naxes, const std::string &extname)
{
    std::vector<std::string> h;
    h.push_back(card("XTENSION", "IMAGE", "image extension", true));
    h.push_back(card_int("BITPIX", -64, "IEEE double precision"));
    h.push_back(card_int("NAXIS", (long long)naxes.size(), "number of axes"));
    for (size_t i = 0; i < naxes.size(); i++)
        h.push_back(card_int("NAXIS" + std::to_string(i + 1), naxes[i], "length of axis " + std::to_string(i + 1)));
    h.push_back(card_int("PCOUNT", 0, "no parameters"));
    h.push_back(card_int("GCOUNT", 1, "one group"));
    h.push_back(card("EXTNAME", extname, "extension name", true));
    return h;
}

// Writes the file; cube(j) returns (pointer, stride) of scale j's cube:
// (coeff_j, 1) for a dynamic per-scale array, element (a, b, g) at
// a + (2bl-1) * (b + 2bl * g); (wav + j, J+1) for the static layout, element
// at (J+1) * (a + (2B-1) * (b + 2B * g)).
template <typename Cube>
int fits_write(const char *fn, const double *scoeff, int J, int B, int N, int bl_scoeff, double alpha,
               const char *comment, Cube cube)
{
    File f(fopen(fn, "wbx"));
    if (!f) {
        if (errno == EEXIST) return set_error(S2DWC_ERROR_FILEIO, "fits_wav_write: file already exists: %s", fn);
        return set_error(S2DWC_ERROR_FILEIO, "fits_wav_write: cannot create %s: %s", fn, strerror(errno));
    }
    int st;
    std::vector<std::string> h;
    h.push_back(card("SIMPLE", "T", "conforms to FITS standard"));
    h.push_back(card_int("BITPIX", -64, "IEEE double precision"));
    h.push_back(card_int("NAXIS", 0, "no data in the primary HDU"));
    h.push_back(card("EXTEND", "T", "extensions follow"));
    comment_cards(h, "  S2DW scale-discretised directional wavelet and scaling coefficients.");
    comment_cards(h, "  Extensions: SCOEFF_REAL, SCOEFF_IMAG, then one WAV cube per scale.");
    {
        char d[32];
        const time_t now = time(nullptr);
        struct tm tmv;
        gmtime_r(&now, &tmv);
        strftime(d, sizeof d, "%Y-%m-%dT%H:%M:%S", &tmv);
        h.push_back(card("DATE", d, "file creation date (YYYY-MM-DDThh:mm:ss UT)", true));
    }
    if (comment && *comment) comment_cards(h, comment);
    h.push_back(card_int("J", J, "No. of scales"));
    h.push_back(card_int("B", B, "Band limit"));
    h.push_back(card_int("N", N, "Azimuthal band limit"));
    h.push_back(card_int("BLSCOEFF", bl_scoeff, "Scaling coefficient band limit"));
    {
        char v[40];
        snprintf(v, sizeof v, "%.8E", alpha);  // 8 decimals, as the reference's ftpkyd call
        h.push_back(card("ALPHA", v, "Alpha"));
    }
    if ((st = write_header(f.get(), h, fn))) return st;
    // scaling coefficients: real, then imaginary parts
    const long long ns = (long long)bl_scoeff * bl_scoeff;
    for (int part = 0; part < 2; part++) {
        if ((st = write_header(f.get(), image_header({bl_scoeff, bl_scoeff}, part ? "SCOEFF_IMAG" : "SCOEFF_REAL"),
                               fn)))
            return st;
        if ((st = write_doubles(f.get(), scoeff + part, ns, 2, fn))) return st;
    }
    const std::vector<int> bl = scale_bl(J, B, alpha);
    for (int j = 0; j <= J; j++) {
        const long long na = 2LL * bl[j] - 1, nb = 2LL * bl[j];
        if ((st = write_header(f.get(), image_header({na, nb, N}, "WAV"), fn))) return st;
        const std::pair<const double *, long long> c = cube(j);
        if (c.second == 1) {
            if ((st = write_doubles(f.get(), c.first, na * nb * N, 1, fn))) return st;
        } else {
            // static layout wav(jj, a, b, g): gather the scale's cube
            std::vector<double> tmp((size_t)(na * nb * N));
            for (long long g = 0; g < N; g++)
                for (long long b = 0; b < nb; b++)
                    for (long long a = 0; a < na; a++)
                        tmp[(size_t)(a + na * (b + nb * g))] = c.first[c.second * (a + (2LL * B - 1) * (b + 2LL * B * g))];
            if ((st = write_doubles(f.get(), tmp.data(), na * nb * N, 1, fn))) return st;
        }
    }
    if (fflush(f.get()) != 0) return set_error(S2DWC_ERROR_FILEIO, "writing %s: %s", fn, strerror(errno));
    return S2DWC_OK;
}

// ---------------------------------------------------------------------------
// FITS reading
// ---------------------------------------------------------------------------
struct Hdu {
    std::map<std::string, std::string> kv;  // keyword -> value field (comment stripped)
    long long data_off = 0, data_bytes = 0;
    int bitpix = 0;
    std::vector<long long> naxes;
};

std::string trim(const std::string &s)
{
    size_t a = s.find_first_not_of(' '), b = s.find_last_not_of(' ');
    return a == std::string::npos ? std::string() : s.substr(a, b - a + 1);
}

// Value field of a card: a quoted string (quotes removed, '' unescaped) or
// the text before a '/' comment.
std::string card_value(const std::string &c)
{
    std::string v = c.size() > 10 ? c.substr(10) : std::string();
    size_t i = v.find_first_not_of(' ');
    if (i != std::string::npos && v[i] == '\'') {
        std::string out;
        for (size_t k = i + 1; k < v.size(); k++) {
            if (v[k] == '\'') {
                if (k + 1 < v.size() && v[k + 1] == '\'') {
                    out += '\'';
                    k++;
                } else {
                    break;
                }
            } else {
                out += v[k];
            }
        }
        return trim(out);
    }
    const size_t s = v.find('/');
    return trim(s == std::string::npos ? v : v.substr(0, s));
}

bool parse_double(const std::string &s0, double *out)
{
    std::string s = s0;
    for (char &ch : s)
        if (ch == 'D' || ch == 'd') ch = 'E';
    if (s.empty()) return false;
    char *end = nullptr;
    errno = 0;
    const double v = strtod(s.c_str(), &end);
    if (end == s.c_str() || errno == ERANGE) return false;
    while (*end == ' ') end++;
    if (*end) return false;
    *out = v;
    return true;
}

bool parse_int(const std::string &s, long long *out)
{
    if (s.empty()) return false;
    char *end = nullptr;
    errno = 0;
    const long long v = strtoll(s.c_str(), &end, 10);
    if (end == s.c_str() || errno == ERANGE) return false;
    while (*end == ' ') end++;
    if (*end) return false;
    *out = v;
    return true;
}

int fits_scan(FILE *f, const char *fn, std::vector<Hdu> &hdus)
{
    if (fseeko(f, 0, SEEK_END) != 0) return set_error(S2DWC_ERROR_FILEIO, "reading %s: %s", fn, strerror(errno));
    const long long size = ftello(f);
    long long pos = 0;
    char blk[BLOCK];
    while (pos < size) {
        Hdu h;
        bool end = false;
        bool first = true;
        while (!end) {
            if (fseeko(f, pos, SEEK_SET) != 0 || fread(blk, 1, BLOCK, f) != (size_t)BLOCK)
                return set_error(S2DWC_ERROR_FILEIO, "reading %s: truncated header at byte %lld", fn, pos);
            pos += BLOCK;
            for (int c = 0; c < BLOCK / CARD; c++) {
                const std::string cd(blk + c * CARD, CARD);
                const std::string key = trim(cd.substr(0, 8));
                if (first) {
                    if (hdus.empty() ? key != "SIMPLE" : key != "XTENSION")
                        return set_error(S2DWC_ERROR_FILEIO, "reading %s: not a FITS %s at byte %lld", fn,
                                         hdus.empty() ? "file" : "extension", pos - BLOCK);
                    first = false;
                }
                if (key == "END") {
                    end = true;
                    break;
                }
                if (cd.size() >= 10 && cd[8] == '=' && cd[9] == ' ' && !h.kv.count(key)) h.kv[key] = card_value(cd);
            }
        }
        long long bp = 0, nax = 0, pc = 0, gc = 1;
        if (!parse_int(h.kv["BITPIX"], &bp) || !parse_int(h.kv["NAXIS"], &nax) || nax < 0 || nax > 999)
            return set_error(S2DWC_ERROR_FILEIO, "reading %s: HDU %zu lacks BITPIX/NAXIS", fn, hdus.size() + 1);
        h.bitpix = (int)bp;
        long long n = nax > 0 ? 1 : 0;
        for (long long i = 1; i <= nax; i++) {
            long long a = 0;
            if (!parse_int(h.kv["NAXIS" + std::to_string(i)], &a) || a < 0)
                return set_error(S2DWC_ERROR_FILEIO, "reading %s: HDU %zu lacks NAXIS%lld", fn, hdus.size() + 1, i);
            h.naxes.push_back(a);
            n *= a;
        }
        if (h.kv.count("PCOUNT")) parse_int(h.kv["PCOUNT"], &pc);
        if (h.kv.count("GCOUNT")) parse_int(h.kv["GCOUNT"], &gc);
        h.data_off = pos;
        h.data_bytes = (std::llabs(bp) / 8) * gc * (pc + n);
        pos += (h.data_bytes + BLOCK - 1) / BLOCK * BLOCK;
        if (pos > size && h.data_bytes > 0) {
            // a data unit may lack its final padding; it may not lack data
            if (h.data_off + h.data_bytes > size)
                return set_error(S2DWC_ERROR_FILEIO, "reading %s: HDU %zu data truncated", fn, hdus.size() + 1);
        }
        hdus.push_back(std::move(h));
    }
    return S2DWC_OK;
}

// Reads the n values of an image HDU as doubles (BSCALE/BZERO applied)
// into out[i * stride].  *anynull: a NaN (floating BITPIX) or a BLANK value
// (integer BITPIX) was read, as CFITSIO's anynull reports.
int fits_read_image(FILE *f, const char *fn, const Hdu &h, double *out, long long n, long long stride, bool *anynull)
{
    const int bytes = std::abs(h.bitpix) / 8;
    if (!(h.bitpix == 8 || h.bitpix == 16 || h.bitpix == 32 || h.bitpix == 64 || h.bitpix == -32 || h.bitpix == -64))
        return set_error(S2DWC_ERROR_FILEIO, "reading %s: unsupported BITPIX %d", fn, h.bitpix);
    double bscale = 1.0, bzero = 0.0;
    auto kv = h.kv;
    if (kv.count("BSCALE")) parse_double(kv["BSCALE"], &bscale);
    if (kv.count("BZERO")) parse_double(kv["BZERO"], &bzero);
    long long blank = 0;
    const bool has_blank = h.bitpix > 0 && kv.count("BLANK") && parse_int(kv["BLANK"], &blank);
    if (fseeko(f, h.data_off, SEEK_SET) != 0) return set_error(S2DWC_ERROR_FILEIO, "reading %s: seek", fn);
    *anynull = false;
    std::vector<unsigned char> buf(1 << 20);
    long long done = 0;
    while (done < n) {
        const long long k = std::min<long long>(n - done, (long long)buf.size() / bytes);
        if (fread(buf.data(), 1, (size_t)(k * bytes), f) != (size_t)(k * bytes))
            return set_error(S2DWC_ERROR_FILEIO, "reading %s: data truncated", fn);
        for (long long i = 0; i < k; i++) {
            uint64_t u = 0;
            for (int b = 0; b < bytes; b++) u = (u << 8) | buf[(size_t)(bytes * i + b)];
            double v;
            bool null = false;
            if (h.bitpix == -64) {
                std::memcpy(&v, &u, 8);
                null = std::isnan(v);
            } else if (h.bitpix == -32) {
                const uint32_t w = (uint32_t)u;
                float x;
                std::memcpy(&x, &w, 4);
                v = x;
                null = std::isnan(x);
            } else {
                long long iv;
                if (h.bitpix == 8) iv = (long long)(uint8_t)u;
                else if (h.bitpix == 16) iv = (long long)(int16_t)(uint16_t)u;
                else if (h.bitpix == 32) iv = (long long)(int32_t)(uint32_t)u;
                else iv = (long long)u;
                null = has_blank && iv == blank;
                v = (double)iv;
            }
            if (null) *anynull = true;
            out[(done + i) * stride] = (bscale == 1.0 && bzero == 0.0) ? v : bzero + bscale * v;
        }
        done += k;
    }
    return S2DWC_OK;
}

struct FitsHeader {
    int J = 0, B = 0, N = 0, bl_scoeff = 0;
    double alpha = 0.0;
};

int fits_open(const char *fn, File &f, std::vector<Hdu> &hdus, FitsHeader &hd)
{
    if (!fn) return set_error(S2DWC_ERROR_ARG_INVALID, "fits_wav_read: null filename");
    f.reset(fopen(fn, "rb"));
    if (!f) return set_error(S2DWC_ERROR_FILEIO, "fits_wav_read: file does not exist: %s", fn);
    int st = fits_scan(f.get(), fn, hdus);
    if (st) return st;
    auto &kv = hdus[0].kv;
    long long J, B, N, bs;
    if (!parse_int(kv["J"], &J) || !parse_int(kv["B"], &B) || !parse_int(kv["N"], &N) ||
        !parse_int(kv["BLSCOEFF"], &bs) || !parse_double(kv["ALPHA"], &hd.alpha))
        return set_error(S2DWC_ERROR_FILEIO, "fits_wav_read: %s lacks J, B, N, BLSCOEFF or ALPHA", fn);
    hd.J = (int)J;
    hd.B = (int)B;
    hd.N = (int)N;
    hd.bl_scoeff = (int)bs;
    if ((st = check_sizes("fits_wav_read", hd.J, hd.B, hd.N, hd.bl_scoeff, hd.alpha)))
        return set_error(S2DWC_ERROR_FILEIO, "fits_wav_read: %s: invalid parameters J=%d B=%d N=%d BLSCOEFF=%d", fn,
                         hd.J, hd.B, hd.N, hd.bl_scoeff);
    // primary + two scaling-coefficient extensions + one per scale (fileio:1333-1340)
    if ((long long)hdus.size() != 1 + 2 + (hd.J + 1LL))
        return set_error(S2DWC_ERROR_FILEIO, "fits_wav_read: %s: invalid number of headers (%zu, expected %d)", fn,
                         hdus.size(), 1 + 2 + (hd.J + 1));
    for (int part = 0; part < 2; part++) {
        const Hdu &h = hdus[1 + part];
        if (h.naxes.size() != 2 || h.naxes[0] != hd.bl_scoeff || h.naxes[1] != hd.bl_scoeff)
            return set_error(S2DWC_ERROR_FILEIO, "fits_wav_read: %s: inconsistent scaling coefficients sizes", fn);
    }
    const std::vector<int> bl = scale_bl(hd.J, hd.B, hd.alpha);
    for (int j = 0; j <= hd.J; j++) {
        const Hdu &h = hdus[3 + j];
        if (h.naxes.size() != 3 || h.naxes[0] != 2LL * bl[j] - 1 || h.naxes[1] != 2LL * bl[j] || h.naxes[2] != hd.N)
            return set_error(S2DWC_ERROR_FILEIO,
                             "fits_wav_read: %s: scale %d cube is not (2bl-1, 2bl, N) = (%d, %d, %d)", fn, j,
                             2 * bl[j] - 1, 2 * bl[j], hd.N);
    }
    return S2DWC_OK;
}

int fits_read_scoeff(FILE *f, const char *fn, const std::vector<Hdu> &hdus, const FitsHeader &hd, double *scoeff)
{
    const long long ns = (long long)hd.bl_scoeff * hd.bl_scoeff;
    for (int part = 0; part < 2; part++) {
        bool anynull = false;
        int st = fits_read_image(f, fn, hdus[1 + part], scoeff + part, ns, 2, &anynull);
        if (st) return st;
    }
    return S2DWC_OK;
}

int require_same(const char *who, const FitsHeader &hd, int J, int B, int N, int bl_scoeff)
{
    if (hd.J != J || hd.B != B || hd.N != N || hd.bl_scoeff != bl_scoeff)
        return set_error(S2DWC_ERROR_SIZE_INVALID,
                         "%s: the file holds J=%d B=%d N=%d bl_scoeff=%d, the buffers are sized for J=%d B=%d N=%d "
                         "bl_scoeff=%d",
                         who, hd.J, hd.B, hd.N, hd.bl_scoeff, J, B, N, bl_scoeff);
    return S2DWC_OK;
}

// ---------------------------------------------------------------------------
// Matlab format
// ---------------------------------------------------------------------------

// Fortran Ew.d output with w = 27, d = 20: [-]0.<20 digits>E<sign><2 digits>,
// or [-]0.<20 digits><sign><3 digits> when the decimal exponent needs three
// digits, right-justified in 27 columns.
std::string fortran_e27_20(double v)
{
    char m[64];
    if (v == 0.0) {
        snprintf(m, sizeof m, "%27s", std::signbit(v) ? "-0.00000000000000000000E+00" : "0.00000000000000000000E+00");
        return m;
    }
    if (!std::isfinite(v)) {
        snprintf(m, sizeof m, "%27s", std::isnan(v) ? "NaN" : (v > 0 ? "Infinity" : "-Infinity"));
        return m;
    }
    char d[64];
    snprintf(d, sizeof d, "%.19E", std::fabs(v));  // d.ddddddddddddddddddddE+xx, 20 significant digits
    const char *e = strchr(d, 'E');
    const int ex = atoi(e + 1) + 1;  // exponent of the 0.ddd form
    std::string digits;
    for (const char *p = d; p < e; p++)
        if (*p != '.') digits += *p;
    std::string s = std::string(v < 0 ? "-" : "") + "0." + digits;
    char tail[16];
    if (std::abs(ex) <= 99) snprintf(tail, sizeof tail, "E%c%02d", ex < 0 ? '-' : '+', std::abs(ex));
    else snprintf(tail, sizeof tail, "%c%03d", ex < 0 ? '-' : '+', std::abs(ex));
    s += tail;
    snprintf(m, sizeof m, "%27s", s.c_str());
    return m;
}

// Reads a Fortran-formatted real: D or E exponent, or a signed exponent
// without a letter (three-digit exponents of the E edit descriptor).
bool parse_fortran_real(const std::string &s0, double *out)
{
    std::string s = trim(s0);
    if (parse_double(s, out)) return true;
    // mantissa followed directly by a signed exponent
    for (size_t i = 1; i < s.size(); i++)
        if ((s[i] == '+' || s[i] == '-') && (isdigit((unsigned char)s[i - 1]) || s[i - 1] == '.')) {
            std::string t = s.substr(0, i) + "E" + s.substr(i);
            return parse_double(t, out);
        }
    return false;
}

std::string base_of(const char *fn)
{
    std::string s(fn);
    if (s.size() >= 2 && s.compare(s.size() - 2, 2, ".m") == 0) s.resize(s.size() - 2);
    return s;
}

template <typename Cube>
int matlab_write(const char *fn, const double *scoeff, int J, int B, int N, int bl_scoeff, double alpha,
                 const char *comment, Cube cube)
{
    const std::string base = base_of(fn);
    const std::string fsc = base + "_scoeff.dat", fwc = base + "_wcoeff.dat";
    std::string name = base;
    const size_t slash = name.find_last_of('/');
    if (slash != std::string::npos) name = name.substr(slash + 1);
    File m(fopen(fn, "wx"));
    if (!m) return set_error(S2DWC_ERROR_FILEIO, "matlab_wav_write: cannot create %s: %s", fn, strerror(errno));
    File s(fopen(fsc.c_str(), "wx"));
    if (!s) return set_error(S2DWC_ERROR_FILEIO, "matlab_wav_write: cannot create %s: %s", fsc.c_str(), strerror(errno));
    File w(fopen(fwc.c_str(), "wx"));
    if (!w) return set_error(S2DWC_ERROR_FILEIO, "matlab_wav_write: cannot create %s: %s", fwc.c_str(), strerror(errno));
    FILE *M = m.get();
    // lines 1-18: header (the reference's reader skips 19 lines, fileio:660-663)
    fprintf(M, "function [J, N, B, bl_scoeff, alpha, scoeff, wcoeff] = %s\n", name.c_str());
    fprintf(M, "%% function [J, N, B, bl_scoeff, alpha, scoeff, wcoeff] = %s\n", name.c_str());
    fprintf(M, "%%\n");
    fprintf(M, "%%  S2DW scale-discretised directional wavelet and scaling coefficients.\n");
    fprintf(M, "%%  Coefficient values are in the two .dat files named below.\n");
    fprintf(M, "%%\n");
    fprintf(M, "%%  This file written by: s2dw_b200 (C)\n");
    fprintf(M, "%%  Comment: %s\n", comment ? comment : "");
    fprintf(M, "%%\n");
    fprintf(M, "%%  Variables:\n");
    fprintf(M, "%%   J: number of wavelet scales minus one (scales 0..J).\n");
    fprintf(M, "%%   B: harmonic band limit.\n");
    fprintf(M, "%%   N: azimuthal band limit.\n");
    fprintf(M, "%%   bl_scoeff: band limit of the scaling coefficients.\n");
    fprintf(M, "%%   alpha: dilation factor between scales.\n");
    fprintf(M, "%%   scoeff(1:bl_scoeff,1:bl_scoeff): scaling coefficients (lower triangle).\n");
    fprintf(M, "%%   wcoeff{1:J+1}(aa,bb,gg): wavelet coefficients of each scale on its (alpha,beta,gamma) grid.\n");
    fprintf(M, "\n");
    // lines 19-24: parameters
    fprintf(M, "%% Size parameters\n");
    fprintf(M, "J         = %27d;\n", J);
    fprintf(M, "N         = %27d;\n", N);
    fprintf(M, "B         = %27d;\n", B);
    fprintf(M, "bl_scoeff = %27d;\n", bl_scoeff);
    fprintf(M, "alpha     = %s;\n", fortran_e27_20(alpha).c_str());
    fprintf(M, "\n");
    fprintf(M, "%% Wavelet coefficient array sizes\n");
    const std::vector<int> bl = scale_bl(J, B, alpha);
    for (int j = 0; j <= J; j++) {
        fprintf(M, "wcoeff_size_aa(%5d) = %15d;\n", j + 1, 2 * bl[j] - 1);
        fprintf(M, "wcoeff_size_bb(%5d) = %15d;\n", j + 1, 2 * bl[j]);
        fprintf(M, "wcoeff_size_gg(%5d) = %15d;\n", j + 1, N);
    }
    fprintf(M, "\n");
    // scaling coefficients: lower triangle, row by row, real then imaginary
    for (int part = 0; part < 2; part++)
        for (int el = 0; el < bl_scoeff; el++)
            for (int mm = 0; mm <= el; mm++)
                fprintf(s.get(), "%s\n", fortran_e27_20(scoeff[2 * ((size_t)el + (size_t)bl_scoeff * mm) + part]).c_str());
    fprintf(M, "%% Scaling coefficients\n");
    fprintf(M, "sc = load('%s');\n", fsc.c_str());
    fprintf(M, "half = numel(sc) / 2;\n");
    fprintf(M, "sc = sc(1:half) + 1i * sc(half+1:end);\n");
    fprintf(M, "scoeff = zeros(bl_scoeff, bl_scoeff);\n");
    fprintf(M, "k = 0;\n");
    fprintf(M, "for el = 1:bl_scoeff\n");
    fprintf(M, "    scoeff(el, 1:el) = sc(k+1:k+el).';\n");
    fprintf(M, "    k = k + el;\n");
    fprintf(M, "end\n");
    fprintf(M, "\n");
    // wavelet coefficients: every scale's cube, first axis fastest
    for (int j = 0; j <= J; j++) {
        const long long na = 2LL * bl[j] - 1, nb = 2LL * bl[j];
        const std::pair<const double *, long long> c = cube(j);
        const long long pa = c.second, pb = c.second == 1 ? na : c.second * (2LL * B - 1),
                        pg = c.second == 1 ? na * nb : c.second * (2LL * B - 1) * 2LL * B;
        for (long long g = 0; g < N; g++)
            for (long long b = 0; b < nb; b++)
                for (long long a = 0; a < na; a++)
                    fprintf(w.get(), "%s\n", fortran_e27_20(c.first[pa * a + pb * b + pg * g]).c_str());
    }
    fprintf(M, "%% Wavelet coefficients\n");
    fprintf(M, "wc = load('%s');\n", fwc.c_str());
    fprintf(M, "wcoeff = cell(1, J+1);\n");
    fprintf(M, "k = 0;\n");
    fprintf(M, "for jj = 1:J+1\n");
    fprintf(M, "    n = wcoeff_size_aa(jj) * wcoeff_size_bb(jj) * wcoeff_size_gg(jj);\n");
    fprintf(M, "    wcoeff{jj} = reshape(wc(k+1:k+n), wcoeff_size_aa(jj), wcoeff_size_bb(jj), wcoeff_size_gg(jj));\n");
    fprintf(M, "    k = k + n;\n");
    fprintf(M, "end\n");
    fprintf(M, "\n");
    if (ferror(M) || ferror(s.get()) || ferror(w.get()))
        return set_error(S2DWC_ERROR_FILEIO, "matlab_wav_write: write error on %s", fn);
    return S2DWC_OK;
}

bool read_line(FILE *f, std::string &line)
{
    line.clear();
    int ch;
    while ((ch = fgetc(f)) != EOF && ch != '\n') line += (char)ch;
    if (!line.empty() && line.back() == '\r') line.pop_back();
    return !(ch == EOF && line.empty());
}

// Value of "name = value;": the text between '=' and the last character,
// as the reference's reader takes it (fileio:666-668).
std::string assigned(const std::string &line)
{
    const size_t e = line.find('=');
    std::string t = trim(line);
    if (e == std::string::npos || t.size() < 2) return std::string();
    const size_t stop = line.find_last_not_of(' ');
    return trim(line.substr(e + 1, stop - e - 1));
}

struct MatHeader {
    int J = 0, B = 0, N = 0, bl_scoeff = 0;
    double alpha = 0.0;
    std::vector<long long> sizes;  // 3 per scale
};

int matlab_header(const char *fn, MatHeader &hd)
{
    if (!fn) return set_error(S2DWC_ERROR_ARG_INVALID, "matlab_wav_read: null filename");
    File f(fopen(fn, "r"));
    if (!f) return set_error(S2DWC_ERROR_FILEIO, "matlab_wav_read: file does not exist: %s", fn);
    std::string line;
    for (int i = 0; i < 19; i++)
        if (!read_line(f.get(), line)) return set_error(S2DWC_ERROR_FILEIO, "matlab_wav_read: %s: short header", fn);
    long long v[4];
    for (int i = 0; i < 4; i++)
        if (!read_line(f.get(), line) || !parse_int(assigned(line), &v[i]))
            return set_error(S2DWC_ERROR_FILEIO, "matlab_wav_read: %s: bad parameter line %d", fn, 20 + i);
    if (!read_line(f.get(), line) || !parse_fortran_real(assigned(line), &hd.alpha))
        return set_error(S2DWC_ERROR_FILEIO, "matlab_wav_read: %s: bad alpha line", fn);
    hd.J = (int)v[0];
    hd.N = (int)v[1];
    hd.B = (int)v[2];
    hd.bl_scoeff = (int)v[3];
    if (check_sizes("matlab_wav_read", hd.J, hd.B, hd.N, hd.bl_scoeff, hd.alpha))
        return set_error(S2DWC_ERROR_FILEIO, "matlab_wav_read: %s: invalid parameters", fn);
    for (int i = 0; i < 2; i++) read_line(f.get(), line);
    const std::vector<int> bl = scale_bl(hd.J, hd.B, hd.alpha);
    for (int j = 0; j <= hd.J; j++) {
        for (int k = 0; k < 3; k++) {
            long long s;
            if (!read_line(f.get(), line) || !parse_int(assigned(line), &s))
                return set_error(S2DWC_ERROR_FILEIO, "matlab_wav_read: %s: bad size line of scale %d", fn, j);
            hd.sizes.push_back(s);
        }
        const long long *s = &hd.sizes[3 * (size_t)j];
        if (s[0] != 2LL * bl[j] - 1 || s[1] != 2LL * bl[j] || s[2] != hd.N)
            return set_error(S2DWC_ERROR_FILEIO, "matlab_wav_read: %s: scale %d sizes are not (2bl-1, 2bl, N)", fn, j);
    }
    return S2DWC_OK;
}

int read_reals(FILE *f, const char *fn, double *dst, long long n, long long stride)
{
    std::string line;
    for (long long i = 0; i < n; i++) {
        if (!read_line(f, line) || !parse_fortran_real(line, &dst[i * stride]))
            return set_error(S2DWC_ERROR_FILEIO, "matlab_wav_read: %s: bad or missing value %lld", fn, i + 1);
    }
    return S2DWC_OK;
}

template <typename Cube>
int matlab_read(const char *fn, const MatHeader &hd, double *scoeff, Cube cube)
{
    const std::string base = base_of(fn);
    const std::string fsc = base + "_scoeff.dat", fwc = base + "_wcoeff.dat";
    File s(fopen(fsc.c_str(), "r"));
    if (!s) return set_error(S2DWC_ERROR_FILEIO, "matlab_wav_read: file does not exist: %s", fsc.c_str());
    const int bs = hd.bl_scoeff;
    for (long long i = 0; i < 2LL * bs * bs; i++) scoeff[i] = 0.0;
    int st;
    for (int part = 0; part < 2; part++)
        for (int el = 0; el < bs; el++)
            for (int mm = 0; mm <= el; mm++)
                if ((st = read_reals(s.get(), fsc.c_str(), scoeff + 2 * ((size_t)el + (size_t)bs * mm) + part, 1, 1)))
                    return st;
    File w(fopen(fwc.c_str(), "r"));
    if (!w) return set_error(S2DWC_ERROR_FILEIO, "matlab_wav_read: file does not exist: %s", fwc.c_str());
    const std::vector<int> bl = scale_bl(hd.J, hd.B, hd.alpha);
    for (int j = 0; j <= hd.J; j++) {
        const long long na = 2LL * bl[j] - 1, nb = 2LL * bl[j];
        const std::pair<double *, long long> c = cube(j);
        const long long pa = c.second, pb = c.second == 1 ? na : c.second * (2LL * hd.B - 1),
                        pg = c.second == 1 ? na * nb : c.second * (2LL * hd.B - 1) * 2LL * hd.B;
        for (long long g = 0; g < hd.N; g++)
            for (long long b = 0; b < nb; b++)
                for (long long a = 0; a < na; a++)
                    if ((st = read_reals(w.get(), fwc.c_str(), c.first + pa * a + pb * b + pg * g, 1, 1))) return st;
    }
    return S2DWC_OK;
}

}  // namespace
}  // namespace s2dw

using namespace s2dw;

extern "C" {

int s2dwc_fileio_fits_wav_write_dynamic(double *const *wav_scales, const double *scoeff, int J, int B, int N,
                                        int bl_scoeff, double alpha, const char *filename, const char *comment)
{
    S2DW_API_TRY
    int st = check_sizes("fits_wav_write_dynamic", J, B, N, bl_scoeff, alpha);
    if (st) return st;
    if (!wav_scales || !filename || (!scoeff && bl_scoeff > 0))
        return set_error(S2DWC_ERROR_ARG_INVALID, "fits_wav_write_dynamic: null pointer");
    for (int j = 0; j <= J; j++)
        if (!wav_scales[j]) return set_error(S2DWC_ERROR_ARG_INVALID, "fits_wav_write_dynamic: scale %d is null", j);
    return fits_write(filename, scoeff, J, B, N, bl_scoeff, alpha, comment,
                      [&](int j) { return std::make_pair((const double *)wav_scales[j], 1LL); });
    S2DW_API_CATCH
}

int s2dwc_fileio_fits_wav_write_static(const double *wav, const double *scoeff, int J, int B, int N, int bl_scoeff,
                                       double alpha, const char *filename, const char *comment)
{
    S2DW_API_TRY
    int st = check_sizes("fits_wav_write_static", J, B, N, bl_scoeff, alpha);
    if (st) return st;
    if (!wav || !filename || (!scoeff && bl_scoeff > 0))
        return set_error(S2DWC_ERROR_ARG_INVALID, "fits_wav_write_static: null pointer");
    return fits_write(filename, scoeff, J, B, N, bl_scoeff, alpha, comment,
                      [&](int j) { return std::make_pair(wav + j, (long long)(J + 1)); });
    S2DW_API_CATCH
}

int s2dwc_fileio_fits_wav_read_header(const char *filename, int *J, int *B, int *N, int *bl_scoeff, double *alpha)
{
    S2DW_API_TRY
    File f;
    std::vector<Hdu> hdus;
    FitsHeader hd;
    int st = fits_open(filename, f, hdus, hd);
    if (st) return st;
    if (J) *J = hd.J;
    if (B) *B = hd.B;
    if (N) *N = hd.N;
    if (bl_scoeff) *bl_scoeff = hd.bl_scoeff;
    if (alpha) *alpha = hd.alpha;
    return S2DWC_OK;
    S2DW_API_CATCH
}

int s2dwc_fileio_fits_wav_read_dynamic(double *const *wav_scales, double *scoeff, int J, int B, int N, int bl_scoeff,
                                       const char *filename)
{
    S2DW_API_TRY
    File f;
    std::vector<Hdu> hdus;
    FitsHeader hd;
    int st = fits_open(filename, f, hdus, hd);
    if (st) return st;
    if ((st = require_same("fits_wav_read_dynamic", hd, J, B, N, bl_scoeff))) return st;
    if (!wav_scales || (!scoeff && bl_scoeff > 0))
        return set_error(S2DWC_ERROR_ARG_INVALID, "fits_wav_read_dynamic: null pointer");
    if (bl_scoeff > 0 && (st = fits_read_scoeff(f.get(), filename, hdus, hd, scoeff))) return st;
    for (int j = 0; j <= J; j++) {
        if (!wav_scales[j]) return set_error(S2DWC_ERROR_ARG_INVALID, "fits_wav_read_dynamic: scale %d is null", j);
        const Hdu &h = hdus[3 + j];
        bool anynull = false;
        if ((st = fits_read_image(f.get(), filename, h, wav_scales[j], h.naxes[0] * h.naxes[1] * h.naxes[2], 1,
                                  &anynull)))
            return st;
        if (anynull)
            return set_error(S2DWC_ERROR_FILEIO, "fits_wav_read_dynamic: null wavelet coefficients read from %s",
                             filename);
    }
    return S2DWC_OK;
    S2DW_API_CATCH
}

int s2dwc_fileio_fits_wav_read_static(double *wav, double *scoeff, int J, int B, int N, int bl_scoeff,
                                      const char *filename)
{
    S2DW_API_TRY
    File f;
    std::vector<Hdu> hdus;
    FitsHeader hd;
    int st = fits_open(filename, f, hdus, hd);
    if (st) return st;
    if ((st = require_same("fits_wav_read_static", hd, J, B, N, bl_scoeff))) return st;
    if (!wav || (!scoeff && bl_scoeff > 0))
        return set_error(S2DWC_ERROR_ARG_INVALID, "fits_wav_read_static: null pointer");
    // the reference zeroes the static array before filling each scale's region
    std::fill(wav, wav + (J + 1LL) * (2LL * B - 1) * 2LL * B * N, 0.0);
    if (bl_scoeff > 0 && (st = fits_read_scoeff(f.get(), filename, hdus, hd, scoeff))) return st;
    for (int j = 0; j <= J; j++) {
        const Hdu &h = hdus[3 + j];
        const long long na = h.naxes[0], nb = h.naxes[1];
        std::vector<double> cube((size_t)(na * nb * N));
        bool anynull = false;
        if ((st = fits_read_image(f.get(), filename, h, cube.data(), na * nb * N, 1, &anynull))) return st;
        if (anynull)
            return set_error(S2DWC_ERROR_FILEIO, "fits_wav_read_static: null wavelet coefficients read from %s",
                             filename);
        for (long long g = 0; g < N; g++)
            for (long long b = 0; b < nb; b++)
                for (long long a = 0; a < na; a++)
                    wav[j + (J + 1LL) * (a + (2LL * B - 1) * (b + 2LL * B * g))] = cube[(size_t)(a + na * (b + nb * g))];
    }
    return S2DWC_OK;
    S2DW_API_CATCH
}

int s2dwc_fileio_matlab_wav_write_dynamic(double *const *wav_scales, const double *scoeff, int J, int B, int N,
                                          int bl_scoeff, double alpha, const char *filename, const char *comment)
{
    S2DW_API_TRY
    int st = check_sizes("matlab_wav_write_dynamic", J, B, N, bl_scoeff, alpha);
    if (st) return st;
    if (!wav_scales || !filename || (!scoeff && bl_scoeff > 0))
        return set_error(S2DWC_ERROR_ARG_INVALID, "matlab_wav_write_dynamic: null pointer");
    for (int j = 0; j <= J; j++)
        if (!wav_scales[j]) return set_error(S2DWC_ERROR_ARG_INVALID, "matlab_wav_write_dynamic: scale %d is null", j);
    return matlab_write(filename, scoeff, J, B, N, bl_scoeff, alpha, comment,
                        [&](int j) { return std::make_pair((const double *)wav_scales[j], 1LL); });
    S2DW_API_CATCH
}

int s2dwc_fileio_matlab_wav_write_static(const double *wav, const double *scoeff, int J, int B, int N, int bl_scoeff,
                                         double alpha, const char *filename, const char *comment)
{
    S2DW_API_TRY
    int st = check_sizes("matlab_wav_write_static", J, B, N, bl_scoeff, alpha);
    if (st) return st;
    if (!wav || !filename || (!scoeff && bl_scoeff > 0))
        return set_error(S2DWC_ERROR_ARG_INVALID, "matlab_wav_write_static: null pointer");
    return matlab_write(filename, scoeff, J, B, N, bl_scoeff, alpha, comment,
                        [&](int j) { return std::make_pair(wav + j, (long long)(J + 1)); });
    S2DW_API_CATCH
}

int s2dwc_fileio_matlab_wav_read_header(const char *filename, int *J, int *B, int *N, int *bl_scoeff, double *alpha)
{
    S2DW_API_TRY
    MatHeader hd;
    int st = matlab_header(filename, hd);
    if (st) return st;
    if (J) *J = hd.J;
    if (B) *B = hd.B;
    if (N) *N = hd.N;
    if (bl_scoeff) *bl_scoeff = hd.bl_scoeff;
    if (alpha) *alpha = hd.alpha;
    return S2DWC_OK;
    S2DW_API_CATCH
}

int s2dwc_fileio_matlab_wav_read_dynamic(double *const *wav_scales, double *scoeff, int J, int B, int N,
                                         int bl_scoeff, const char *filename)
{
    S2DW_API_TRY
    MatHeader hd;
    int st = matlab_header(filename, hd);
    if (st) return st;
    if (hd.J != J || hd.B != B || hd.N != N || hd.bl_scoeff != bl_scoeff)
        return set_error(S2DWC_ERROR_SIZE_INVALID, "matlab_wav_read_dynamic: the file holds J=%d B=%d N=%d "
                         "bl_scoeff=%d", hd.J, hd.B, hd.N, hd.bl_scoeff);
    if (!wav_scales || (!scoeff && bl_scoeff > 0))
        return set_error(S2DWC_ERROR_ARG_INVALID, "matlab_wav_read_dynamic: null pointer");
    for (int j = 0; j <= J; j++)
        if (!wav_scales[j]) return set_error(S2DWC_ERROR_ARG_INVALID, "matlab_wav_read_dynamic: scale %d is null", j);
    return matlab_read(filename, hd, scoeff, [&](int j) { return std::make_pair(wav_scales[j], 1LL); });
    S2DW_API_CATCH
}

int s2dwc_fileio_matlab_wav_read_static(double *wav, double *scoeff, int J, int B, int N, int bl_scoeff,
                                        const char *filename)
{
    S2DW_API_TRY
    MatHeader hd;
    int st = matlab_header(filename, hd);
    if (st) return st;
    if (hd.J != J || hd.B != B || hd.N != N || hd.bl_scoeff != bl_scoeff)
        return set_error(S2DWC_ERROR_SIZE_INVALID, "matlab_wav_read_static: the file holds J=%d B=%d N=%d "
                         "bl_scoeff=%d", hd.J, hd.B, hd.N, hd.bl_scoeff);
    if (!wav || (!scoeff && bl_scoeff > 0))
        return set_error(S2DWC_ERROR_ARG_INVALID, "matlab_wav_read_static: null pointer");
    std::fill(wav, wav + (J + 1LL) * (2LL * B - 1) * 2LL * B * N, 0.0);
    return matlab_read(filename, hd, scoeff, [&](int j) { return std::make_pair(wav + j, (long long)(J + 1)); });
    S2DW_API_CATCH
}

}  // extern "C"
