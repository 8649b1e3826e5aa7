// deck_io.cpp -- native reader/writer of the reference's Tecplot-ASCII deck.
//
// Format (writer v1.9/codes/main_v1.9.f90:759-773, reader :213-239):
//   TITLE ="<time F20.10><nstep I9>"
//    Variables ="x","y","z","Rho","U","V","W","E","T","P"
//   ZONE k=<I3>,j=<I3>,i=<I3>,DATAPACKING="POINT"
// then for k, for j: one blank line before each k block and each j block,
// and nP1 records 3(1X,F10.6),7(1X,E22.15) = x,y,z,rho,u,v,w,E,T,p.
// The field var(1:nP1,1:nP2,1:nP3,1:7) is column-major (i fastest).
// Formatting and parsing run on host threads; this file never touches the GPU.
#include "chanrhs.h"

#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

namespace {

std::string g_io_error;

int io_fail(const std::string &m)
{
    g_io_error = m;
    return CHAN_EIO;
}

int nthreads_of(int32_t n)
{
    if (n > 0) return n;
    unsigned h = std::thread::hardware_concurrency();
    return h ? (int)h : 1;
}

template <class F>
void parallel_for(int n, int nth, F f)
{
    if (nth <= 1 || n <= 1) {
        for (int k = 0; k < n; k++) f(k);
        return;
    }
    std::vector<std::thread> th;
    const int per = (n + nth - 1) / nth;
    for (int t = 0; t < nth; t++) {
        const int a = t * per, b = a + per < n ? a + per : n;
        if (a >= b) break;
        th.emplace_back([=, &f] {
            for (int k = a; k < b; k++) f(k);
        });
    }
    for (auto &x : th) x.join();
}

// Fortran E22.15: [-]0.ddddddddddddddd E+xx, right-justified in 22 columns
void fmt_e22_15(double x, char *out)
{
    char body[40];
    if (x != x || std::isinf(x)) {
        snprintf(out, 23, "%22s", x != x ? "NaN" : (x < 0 ? "-Infinity" : "Infinity"));
        return;
    }
    const bool neg = std::signbit(x) && x != 0.0;
    if (x == 0.0) {
        strcpy(body, "0.000000000000000E+00");
    } else {
        char s[40];
        snprintf(s, sizeof(s), "%.14E", std::fabs(x));  // d.ddddddddddddddE+XX
        char digits[16];
        digits[0] = s[0];
        memcpy(digits + 1, s + 2, 14);
        digits[15] = 0;
        const int e = atoi(s + 17) + 1;
        if (e >= -99 && e <= 99)
            snprintf(body, sizeof(body), "0.%sE%c%02d", digits, e < 0 ? '-' : '+', e < 0 ? -e : e);
        else
            snprintf(body, sizeof(body), "0.%s%c%03d", digits, e < 0 ? '-' : '+', e < 0 ? -e : e);
    }
    char full[48];
    snprintf(full, sizeof(full), "%s%s", neg ? "-" : "", body);
    const size_t n = strlen(full) < 22 ? strlen(full) : 22;
    memset(out, ' ', 22 - n);
    memcpy(out + 22 - n, full, n);
    out[22] = 0;
}

// one Fortran real field: accepts E/D exponents and the 3-digit form without a letter
bool parse_real(const char *p, const char *end, double *v, const char **next)
{
    while (p < end && (*p == ' ' || *p == '\t')) p++;
    if (p >= end) return false;
    char buf[64];
    int n = 0;
    while (p < end && *p != ' ' && *p != '\t' && *p != '\n' && *p != '\r' && n < 63) {
        char c = *p++;
        buf[n++] = (c == 'D' || c == 'd') ? 'E' : c;
    }
    buf[n] = 0;
    if (n == 0) return false;
    char *e = nullptr;
    errno = 0;
    double x = strtod(buf, &e);
    if (e == buf) return false;
    if (*e == '+' || *e == '-') {  // 0.123+100
        char *e2 = nullptr;
        long ex = strtol(e, &e2, 10);
        if (e2 == e || *e2) return false;
        x = x * std::pow(10.0, (double)ex);
    } else if (*e) {
        return false;
    }
    *v = x;
    *next = p;
    return true;
}

}  // namespace

extern "C" {

const char *chan_io_last_error(void) { return g_io_error.c_str(); }

int chan_deck_write(const char *path, const int32_t *nP, const double *var, const double *x1, const double *x2,
                    const double *x3, double time, int64_t nstep, int32_t nthreads)
{
    if (!path || !nP || !var || !x1 || !x2 || !x3) return CHAN_EINVAL;
    const long long n1 = nP[0], n2 = nP[1], n3 = nP[2];
    if (n1 < 1 || n2 < 1 || n3 < 1) return CHAN_EINVAL;
    const long long N = n1 * n2 * n3;
    constexpr int REC = 3 * 11 + 7 * 23 + 1 + 64;   // one record, its newline, margin for wide coordinates
    FILE *f = fopen(path, "wb");
    if (!f) return io_fail(std::string("cannot open ") + path + ": " + strerror(errno));
    fprintf(f, "TITLE =\"%20.10f%9lld\"\n", time, (long long)nstep);
    fprintf(f, " Variables =\"x\",\"y\",\"z\",\"Rho\",\"U\",\"V\",\"W\",\"E\",\"T\",\"P\"\n");
    fprintf(f, "ZONE k=%3lld,j=%3lld,i=%3lld,DATAPACKING=\"POINT\"\n", n3, n2, n1);
    const int nth = nthreads_of(nthreads);
    // format k-planes in batches so the text buffer stays bounded
    const long long plane_bytes = n2 * (1 + n1 * REC) + 1;
    const int batch = (int)std::max<long long>(1, std::min<long long>(n3, (512LL << 20) / plane_bytes));
    std::vector<char> buf((size_t)batch * plane_bytes);
    std::vector<long long> used(batch);
    int rc = CHAN_OK;
    for (long long k0 = 0; k0 < n3 && rc == CHAN_OK; k0 += batch) {
        const int nb = (int)std::min<long long>(batch, n3 - k0);
        parallel_for(nb, nth, [&](int kb) {
            const long long k = k0 + kb;
            char *o = buf.data() + (size_t)kb * plane_bytes;
            char *p = o;
            *p++ = '\n';
            for (long long j = 0; j < n2; j++) {
                *p++ = '\n';
                for (long long i = 0; i < n1; i++) {
                    p += sprintf(p, " %10.6f %10.6f %10.6f", x1[i], x2[j], x3[k]);
                    const long long r = (k * n2 + j) * n1 + i;
                    for (int m = 0; m < 7; m++) {
                        *p++ = ' ';
                        fmt_e22_15(var[(size_t)m * N + r], p);
                        p += 22;
                    }
                    *p++ = '\n';
                }
            }
            used[kb] = p - o;
        });
        for (int kb = 0; kb < nb; kb++)
            if (fwrite(buf.data() + (size_t)kb * plane_bytes, 1, (size_t)used[kb], f) != (size_t)used[kb]) {
                rc = io_fail(std::string("write failed: ") + path);
                break;
            }
    }
    if (fclose(f) != 0 && rc == CHAN_OK) rc = io_fail(std::string("close failed: ") + path);
    return rc;
}

int chan_deck_read(const char *path, const int32_t *nP, double *var, double *x1, double *x2, double *x3,
                   double *time, int64_t *nstep, int32_t nthreads)
{
    if (!path || !nP || !var) return CHAN_EINVAL;
    const long long n1 = nP[0], n2 = nP[1], n3 = nP[2];
    const long long N = n1 * n2 * n3;
    FILE *f = fopen(path, "rb");
    if (!f) return io_fail(std::string("cannot open ") + path + ": " + strerror(errno));
    fseek(f, 0, SEEK_END);
    const long long sz = ftell(f);
    fseek(f, 0, SEEK_SET);
    std::vector<char> text((size_t)sz + 1);
    const size_t got = fread(text.data(), 1, (size_t)sz, f);
    fclose(f);
    if ((long long)got != sz) return io_fail(std::string("read failed: ") + path);
    text[sz] = '\n';
    const char *b = text.data(), *e = b + sz;
    // header: 8X,F20.10,I9
    const char *eol = (const char *)memchr(b, '\n', sz);
    if (!eol || eol - b < 37) return io_fail("bad header line");
    {
        char t[32], s[16];
        memcpy(t, b + 8, 20); t[20] = 0;
        memcpy(s, b + 28, 9); s[9] = 0;
        char *q;
        const double tv = strtod(t, &q);
        if (q == t) return io_fail("bad time in header");
        if (time) *time = tv;
        if (nstep) *nstep = strtoll(s, nullptr, 10);
    }
    const char *p = eol + 1;
    for (int h = 0; h < 2; h++) {
        const char *x = (const char *)memchr(p, '\n', e - p);
        if (!x) return io_fail("missing header lines");
        p = x + 1;
    }
    // offsets of the data records (non-blank lines)
    std::vector<const char *> rec;
    rec.reserve((size_t)N);
    while (p < e) {
        const char *x = (const char *)memchr(p, '\n', e - p + 1);
        if (!x) x = e;
        bool blank = true;
        for (const char *c = p; c < x; c++)
            if (*c != ' ' && *c != '\r' && *c != '\t') { blank = false; break; }
        if (!blank) rec.push_back(p);
        p = x + 1;
    }
    auto where = [&](long long r) {
        char m[160];
        const long long i = r % n1, j = (r / n1) % n2, k = r / (n1 * n2);
        snprintf(m, sizeof(m), "Error in reading combined input file at %lld %lld %lld", i + 1, j + 1, k + 1);
        return std::string(m);
    };
    if ((long long)rec.size() < N) return io_fail(where((long long)rec.size()) + " (file ends)");
    std::vector<long long> bad(nthreads_of(nthreads) + 1, -1);
    const int nth = nthreads_of(nthreads);
    const long long per = (N + nth - 1) / nth;
    parallel_for(nth, nth, [&](int t) {
        const long long a = t * per, z = std::min(N, a + per);
        for (long long r = a; r < z; r++) {
            const char *q = rec[(size_t)r];
            const char *end = (const char *)memchr(q, '\n', e - q + 1);
            double v[10];
            for (int c = 0; c < 10; c++)
                if (!parse_real(q, end, &v[c], &q)) { bad[t] = r; return; }
            const long long i = r % n1, j = (r / n1) % n2, k = r / (n1 * n2);
            if (x1 && j == 0 && k == 0) x1[i] = v[0];
            if (x2 && i == 0 && k == 0) x2[j] = v[1];
            if (x3 && i == 0 && j == 0) x3[k] = v[2];
            for (int m = 0; m < 7; m++) var[(size_t)m * N + r] = v[3 + m];
        }
    });
    long long first = -1;
    for (long long r : bad)
        if (r >= 0 && (first < 0 || r < first)) first = r;
    if (first >= 0) return io_fail(where(first));
    return CHAN_OK;
}

}  // extern "C"
