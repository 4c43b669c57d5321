// Grid ingestion for the drivers' input step.  code.f90:36-56 and
// mom6_code.f90:95-117 read five files of point_count values each (areas,
// x, y, z, ssh), one value per line, with Fortran list-directed reads, one
// READ statement per value.  sal_read_values parses such a file with every
// host thread, or reads the raw little-endian float64 form (".f64") that
// sal_write_values writes.
#include <cerrno>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/salgpu.h"

#ifdef _OPENMP
#include <omp.h>
#endif

namespace sal {
int set_error(int code, const std::string &msg);  // capi.cpp
}

using sal::set_error;

namespace {

bool ends_with(const std::string &s, const char *suffix) {
    const size_t n = std::strlen(suffix);
    return s.size() >= n && s.compare(s.size() - n, n, suffix) == 0;
}

int read_file(const char *path, std::vector<char> *buf) {
    FILE *f = std::fopen(path, "rb");
    if (!f) return set_error(SAL_EINVAL, std::string("cannot open ") + path + ": " + std::strerror(errno));
    std::fseek(f, 0, SEEK_END);
    const long len = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    buf->resize((size_t)(len > 0 ? len : 0) + 1);
    const size_t got = len > 0 ? std::fread(buf->data(), 1, (size_t)len, f) : 0;
    std::fclose(f);
    if ((long)got != len) return set_error(SAL_EINVAL, std::string("short read of ") + path);
    (*buf)[got] = '\0';
    buf->resize(got + 1);
    return SAL_OK;
}

// One value of a list-directed record: leading blanks, an optional sign, digits
// with an optional point, an optional exponent with E, D or Q (or a bare sign,
// as in 1.0-300), then blanks, a comma or the end of the line.
bool parse_value(const char *b, const char *e, double *out) {
    char tmp[64];
    while (b < e && (*b == ' ' || *b == '\t' || *b == '\r')) ++b;
    while (e > b && (e[-1] == ' ' || e[-1] == '\t' || e[-1] == '\r' || e[-1] == ',')) --e;
    const size_t n = (size_t)(e - b);
    if (n == 0 || n >= sizeof(tmp) - 1) return false;
    size_t k = 0;
    bool digits = false;
    for (size_t i = 0; i < n; ++i) {
        char c = b[i];
        if (c == 'd' || c == 'D' || c == 'q' || c == 'Q') c = 'E';
        // Fortran may drop the exponent letter: 1.0-300 means 1.0E-300
        if ((c == '+' || c == '-') && i > 0 && digits && b[i - 1] != 'E' && b[i - 1] != 'e' && b[i - 1] != 'D' &&
            b[i - 1] != 'd' && b[i - 1] != 'Q' && b[i - 1] != 'q')
            tmp[k++] = 'E';
        if (c >= '0' && c <= '9') digits = true;
        tmp[k++] = c;
    }
    tmp[k] = '\0';
    char *end = nullptr;
    errno = 0;
    const double v = std::strtod(tmp, &end);
    if (end == tmp || *end != '\0') return false;
    *out = v;
    return true;
}

}  // namespace

extern "C" int sal_read_values(const char *path, int64_t count, double *out) {
    if (!path || (count > 0 && !out)) return set_error(SAL_EINVAL, "null argument");
    if (count < 0) return set_error(SAL_EINVAL, "negative count");
    const std::string p(path);
    std::vector<char> buf;
    int rc = read_file(path, &buf);
    if (rc) return rc;
    const size_t len = buf.size() - 1;
    if (ends_with(p, ".f64")) {
        if (len < (size_t)count * sizeof(double))
            return set_error(SAL_EINVAL, p + " holds fewer than " + std::to_string(count) + " float64 values");
        if (count) std::memcpy(out, buf.data(), (size_t)count * sizeof(double));
        return SAL_OK;
    }
    // line starts, found per block in parallel and joined in order
    const char *s = buf.data();
    int nth = 1;
#ifdef _OPENMP
    nth = omp_get_max_threads();
#endif
    const size_t blk = (len + (size_t)nth - 1) / (size_t)nth + 1;
    std::vector<std::vector<size_t>> starts((size_t)nth);
#pragma omp parallel for schedule(static) num_threads(nth)
    for (int t = 0; t < nth; ++t) {
        const size_t lo = (size_t)t * blk, hi = std::min(len, lo + blk);
        for (size_t i = lo; i < hi; ++i)
            if (i == 0 || s[i - 1] == '\n') starts[(size_t)t].push_back(i);
    }
    std::vector<size_t> line;
    for (auto &v : starts) line.insert(line.end(), v.begin(), v.end());
    // blank lines hold no value (list-directed reads skip them)
    std::vector<size_t> rec;
    rec.reserve(line.size());
    for (size_t i = 0; i < line.size(); ++i) {
        const size_t e = i + 1 < line.size() ? line[i + 1] : len;
        bool blank = true;
        for (size_t j = line[i]; j < e && blank; ++j) blank = s[j] == ' ' || s[j] == '\t' || s[j] == '\r' || s[j] == '\n';
        if (!blank) rec.push_back(i);
    }
    if ((int64_t)rec.size() < count)
        return set_error(SAL_EINVAL, p + " holds " + std::to_string(rec.size()) + " values, fewer than " +
                                         std::to_string(count));
    int64_t bad = -1;
#pragma omp parallel for schedule(static) num_threads(nth)
    for (int64_t k = 0; k < count; ++k) {
        const size_t i = rec[(size_t)k];
        const size_t b = line[i], e = i + 1 < line.size() ? line[i + 1] : len;
        size_t stop = e;
        while (stop > b && (s[stop - 1] == '\n')) --stop;
        if (!parse_value(s + b, s + stop, out + k)) {
#pragma omp critical
            if (bad < 0 || k < bad) bad = k;
        }
    }
    if (bad >= 0) return set_error(SAL_EINVAL, p + ": value " + std::to_string(bad + 1) + " is not a number");
    return SAL_OK;
}

extern "C" int sal_write_values(const char *path, int64_t count, const double *values) {
    if (!path || (count > 0 && !values)) return set_error(SAL_EINVAL, "null argument");
    if (count < 0) return set_error(SAL_EINVAL, "negative count");
    FILE *f = std::fopen(path, "wb");
    if (!f) return set_error(SAL_EINVAL, std::string("cannot open ") + path + ": " + std::strerror(errno));
    const size_t put = count ? std::fwrite(values, sizeof(double), (size_t)count, f) : 0;
    const bool ok = std::fclose(f) == 0 && (int64_t)put == count;
    if (!ok) return set_error(SAL_EINVAL, std::string("short write of ") + path);
    return SAL_OK;
}
