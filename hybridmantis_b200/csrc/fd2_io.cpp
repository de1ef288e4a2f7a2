// fd2_io.cpp -- input file, output files and EDE stream files.
//
// Host-only C++.  Formats follow the reference:
//   hybridMANTIS_input.in   main/hybridMANTIS_penEasy.f:190-229 (reader),
//                           :290-299 (raw strings kept for file names)
//   myimage_<tags>.dat      main/hybridMANTIS_tallyEnergyDepositionEvents.f:
//   detected_<tags>.dat     418-458 (names, (1x,F12.4) blocks, (1x,I8) rows)
//   EDE text rows           the tally's event write (3(1x,1pe16.9),1x,1pe12.4,i8)
//                           in cm / eV / 1-based history, :173-174
#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include "fd2.h"
#include "fd2_host.h"

namespace {

// Fortran list-directed reals accept a 'd' exponent.
bool parse_real(const std::string &tok, double *out)
{
    std::string t = tok;
    for (char &c : t)
        if (c == 'd' || c == 'D') c = 'e';
    char *end = nullptr;
    errno = 0;
    const double v = std::strtod(t.c_str(), &end);
    if (end == t.c_str() || *end != '\0' || errno == ERANGE) return false;
    *out = v;
    return true;
}

bool parse_int(const std::string &tok, int32_t *out)
{
    char *end = nullptr;
    errno = 0;
    const long v = std::strtol(tok.c_str(), &end, 10);
    if (end == tok.c_str() || *end != '\0' || errno == ERANGE || v < INT32_MIN || v > INT32_MAX) return false;
    *out = (int32_t)v;
    return true;
}

void set_tag(char dst[11], const std::string &raw)
{
    std::memset(dst, 0, 11);
    std::strncpy(dst, raw.c_str(), 10);
}

// "%g"-style raw strings for params built without a file.
std::string num_tag(double v)
{
    char b[64];
    std::snprintf(b, sizeof b, "%g", v);
    return b;
}

}  // namespace

extern "C" {

fd2_status fd2_parse_input_file(const char *path, fd2_params *out)
{
    if (!path || !out) return FD2_ERR_INVALID_ARGUMENT;
    FILE *f = std::fopen(path, "r");
    if (!f) return FD2_ERR_IO;
    std::vector<std::string> vals;
    char line[4096];
    while (std::fgets(line, sizeof line, f)) {
        const char *s = line;
        while (*s == ' ' || *s == '\t') ++s;
        if (*s == '#' || *s == '\0' || *s == '\n' || *s == '\r') continue;
        const char *e = s;
        while (*e && *e != ' ' && *e != '\t' && *e != '\n' && *e != '\r') ++e;
        vals.emplace_back(s, e);
    }
    std::fclose(f);
    if (vals.size() < 24) return FD2_ERR_PARSE;
    fd2_params p;
    std::memset(&p, 0, sizeof p);
    bool ok = parse_int(vals[0], &p.num_hist) && parse_int(vals[1], &p.min_photons) &&
              parse_int(vals[2], &p.max_photons) && parse_int(vals[3], &p.num_bins) &&
              parse_real(vals[4], &p.det_x) && parse_real(vals[5], &p.det_y) &&
              parse_real(vals[6], &p.det_height) && parse_real(vals[7], &p.radius) &&
              parse_real(vals[8], &p.n_col) && parse_real(vals[9], &p.n_gap) &&
              parse_real(vals[10], &p.top_absfrac) && parse_real(vals[11], &p.bulk_abs) &&
              parse_real(vals[12], &p.beta) && parse_real(vals[13], &p.d_min) &&
              parse_real(vals[14], &p.d_max) && parse_real(vals[15], &p.lb_x) &&
              parse_real(vals[16], &p.lb_y) && parse_real(vals[17], &p.ub_x) &&
              parse_real(vals[18], &p.ub_y) && parse_real(vals[19], &p.yield) &&
              parse_int(vals[20], &p.pixel) && parse_real(vals[21], &p.sensor_refl) &&
              parse_int(vals[22], &p.run_gpu) && parse_int(vals[23], &p.machine);
    if (!ok) return FD2_ERR_PARSE;
    // raw strings for the output names, in the reference's order
    const int idx[10] = {6, 7, 10, 11, 12, 14, 21, 19, 20, 23};
    for (int k = 0; k < 10; ++k) set_tag(p.tag[k], vals[idx[k]]);
    *out = p;
    return FD2_OK;
}

fd2_status fd2_params_fill_tags(fd2_params *p)
{
    if (!p) return FD2_ERR_INVALID_ARGUMENT;
    const double v[10] = {p->det_height, p->radius, p->top_absfrac, p->bulk_abs, p->beta,
                          p->d_max, p->sensor_refl, p->yield, (double)p->pixel, (double)p->machine};
    for (int k = 0; k < 10; ++k)
        if (p->tag[k][0] == '\0') set_tag(p->tag[k], num_tag(v[k]));
    return FD2_OK;
}

fd2_status fd2_params_to_geometry(const fd2_params *p, fd2_geometry *g)
{
    if (!p || !g) return FD2_ERR_INVALID_ARGUMENT;
    std::memset(g, 0, sizeof *g);
    g->det_x = p->det_x;
    g->det_y = p->det_y;
    g->det_height = p->det_height;
    g->radius = p->radius;
    g->n_col = p->n_col;
    g->n_gap = p->n_gap;
    g->top_absfrac = p->top_absfrac;
    g->bulk_abs = p->bulk_abs;
    g->beta = p->beta;
    g->d_min = p->d_min;
    g->d_max = p->d_max;
    g->lb_x = p->lb_x;
    g->lb_y = p->lb_y;
    g->ub_x = p->ub_x;
    g->ub_y = p->ub_y;
    g->sensor_refl = p->sensor_refl;
    g->pixel = p->pixel;
    return FD2_OK;
}

fd2_status fd2_prf_dims(const fd2_geometry *g, int32_t *xdim, int32_t *ydim)
{
    if (!g || !xdim || !ydim || g->pixel <= 0) return FD2_ERR_INVALID_ARGUMENT;
    // float arithmetic of the reference's driver (cuda:184-185)
    const float px = (float)g->pixel;
    const float fx = std::ceil(((float)g->ub_x - (float)g->lb_x) / px);
    const float fy = std::ceil(((float)g->ub_y - (float)g->lb_y) / px);
    if (!(fx >= 1.0f) || !(fy >= 1.0f) || fx > 65536.0f || fy > 65536.0f) return FD2_ERR_INVALID_ARGUMENT;
    *xdim = (int32_t)fx;
    *ydim = (int32_t)fy;
    return FD2_OK;
}

void fd2_free_events(fd2_events *ev)
{
    if (!ev) return;
    std::free(ev->x_um);
    std::free(ev->y_um);
    std::free(ev->z_um);
    std::free(ev->e_ev);
    std::free(ev->hist);
    std::free(ev->geom);
    std::free(ev->geometries);
    std::memset(ev, 0, sizeof *ev);
}

fd2_status fd2_read_events_text(const char *path, fd2_events *out)
{
    if (!path || !out) return FD2_ERR_INVALID_ARGUMENT;
    std::vector<float> x, y, z, e;
    std::vector<int32_t> h;
    int32_t max_hist = 0;
    const fd2_status st = fd2host::stream_events_text(
        path, 1 << 16,
        [&](const double *xc, const double *yc, const double *zc, const double *de, const int32_t *hh, int64_t n) {
            for (int64_t i = 0; i < n; ++i) {
                // cm -> um as the reference's host driver does (double * 10000.0f)
                x.push_back((float)(xc[i] * (double)10000.0f));
                y.push_back((float)(yc[i] * (double)10000.0f));
                z.push_back((float)(zc[i] * (double)10000.0f));
                e.push_back((float)de[i]);
                h.push_back(hh[i]);
                if (hh[i] > max_hist) max_hist = hh[i];
            }
            return FD2_OK;
        });
    if (st != FD2_OK) return st;
    return fd2host::events_from_vectors(x, y, z, e, h, max_hist, out);
}

fd2_status fd2_write_events_text(const char *path, const fd2_events *ev)
{
    if (!path || !ev || ev->n < 0) return FD2_ERR_INVALID_ARGUMENT;
    FILE *f = std::fopen(path, "w");
    if (!f) return FD2_ERR_IO;
    for (int64_t i = 0; i < ev->n; ++i) {
        std::fprintf(f, " %16.9E %16.9E %16.9E %12.4E%8d\n", ev->x_um[i] / 10000.0, ev->y_um[i] / 10000.0,
                     ev->z_um[i] / 10000.0, (double)ev->e_ev[i], ev->hist[i]);
    }
    return std::fclose(f) == 0 ? FD2_OK : FD2_ERR_IO;
}

static const char kBinMagic[8] = {'F', 'D', '2', 'E', 'V', 'T', '0', '1'};

fd2_status fd2_write_events_binary(const char *path, const fd2_events *ev)
{
    if (!path || !ev || ev->n < 0) return FD2_ERR_INVALID_ARGUMENT;
    FILE *f = std::fopen(path, "wb");
    if (!f) return FD2_ERR_IO;
    const int64_t n = ev->n;
    const int32_t has_geom = ev->geom ? 1 : 0;
    bool ok = std::fwrite(kBinMagic, 1, 8, f) == 8 && std::fwrite(&n, 8, 1, f) == 1 &&
              std::fwrite(&ev->num_hist, 4, 1, f) == 1 && std::fwrite(&has_geom, 4, 1, f) == 1;
    ok = ok && std::fwrite(ev->x_um, 4, (size_t)n, f) == (size_t)n && std::fwrite(ev->y_um, 4, (size_t)n, f) == (size_t)n &&
         std::fwrite(ev->z_um, 4, (size_t)n, f) == (size_t)n && std::fwrite(ev->e_ev, 4, (size_t)n, f) == (size_t)n &&
         std::fwrite(ev->hist, 4, (size_t)n, f) == (size_t)n;
    if (ok && has_geom) ok = std::fwrite(ev->geom, 2, (size_t)n, f) == (size_t)n;
    const int rc = std::fclose(f);
    return ok && rc == 0 ? FD2_OK : FD2_ERR_IO;
}

fd2_status fd2_read_events_binary(const char *path, fd2_events *out)
{
    if (!path || !out) return FD2_ERR_INVALID_ARGUMENT;
    fd2_events ev;
    std::memset(&ev, 0, sizeof ev);
    int64_t at = 0;
    const fd2_status st = fd2host::stream_events_binary(
        path, 1 << 20,
        [&](const fd2host::BinHeader &hd) {
            ev.n = hd.n;
            ev.num_hist = hd.num_hist;
            ev.num_geom = 1;
            const size_t N = (size_t)hd.n ? (size_t)hd.n : 1;
            ev.x_um = (float *)std::malloc(4 * N);
            ev.y_um = (float *)std::malloc(4 * N);
            ev.z_um = (float *)std::malloc(4 * N);
            ev.e_ev = (float *)std::malloc(4 * N);
            ev.hist = (int32_t *)std::malloc(4 * N);
            if (hd.has_geom) ev.geom = (uint16_t *)std::malloc(2 * N);
            if (!ev.x_um || !ev.y_um || !ev.z_um || !ev.e_ev || !ev.hist || (hd.has_geom && !ev.geom))
                return FD2_ERR_OUT_OF_MEMORY;
            return FD2_OK;
        },
        [&](const float *x, const float *y, const float *z, const float *e, const int32_t *h, const uint16_t *g,
            int64_t n) {
            std::memcpy(ev.x_um + at, x, 4 * (size_t)n);
            std::memcpy(ev.y_um + at, y, 4 * (size_t)n);
            std::memcpy(ev.z_um + at, z, 4 * (size_t)n);
            std::memcpy(ev.e_ev + at, e, 4 * (size_t)n);
            std::memcpy(ev.hist + at, h, 4 * (size_t)n);
            if (g && ev.geom) std::memcpy(ev.geom + at, g, 2 * (size_t)n);
            at += n;
            return FD2_OK;
        });
    if (st != FD2_OK) {
        fd2_free_events(&ev);
        return st;
    }
    *out = ev;
    return FD2_OK;
}

fd2_status fd2_write_output_files(const fd2_params *p, const fd2_geometry *g, const uint64_t *image, int32_t xdim,
                                  int32_t ydim, const int32_t *phs, int32_t num_bins, double num_hist, const char *dir,
                                  const char *suffix)
{
    if (!p || !g || !image || !phs || !dir || xdim <= 0 || ydim <= 0 || num_bins <= 0 || !(num_hist > 0.0))
        return FD2_ERR_INVALID_ARGUMENT;
    fd2_params q = *p;
    fd2_params_fill_tags(&q);
    std::string base(dir);
    if (!base.empty() && base.back() != '/') base += '/';
    std::string prf_name = fd2host::output_name(q, "myimage_");
    std::string det_name = fd2host::output_name(q, "detected_");
    if (suffix && *suffix) {
        prf_name = prf_name.substr(0, prf_name.size() - 4) + suffix + ".dat";
        det_name = det_name.substr(0, det_name.size() - 4) + suffix + ".dat";
    }
    fd2_status st = fd2host::write_new_file(base + prf_name, fd2host::format_prf(image, xdim, ydim, *g, num_hist));
    if (st != FD2_OK) return st;
    return fd2host::write_new_file(base + det_name, fd2host::format_phs(phs, num_bins));
}

}  // extern "C"

namespace fd2host {

fd2_status events_from_vectors(const std::vector<float> &x, const std::vector<float> &y, const std::vector<float> &z,
                               const std::vector<float> &e, const std::vector<int32_t> &h, int32_t num_hist,
                               fd2_events *out)
{
    fd2_events ev;
    std::memset(&ev, 0, sizeof ev);
    const size_t n = x.size();
    const size_t N = n ? n : 1;
    ev.n = (int64_t)n;
    ev.num_hist = num_hist;
    ev.num_geom = 1;
    ev.x_um = (float *)std::malloc(4 * N);
    ev.y_um = (float *)std::malloc(4 * N);
    ev.z_um = (float *)std::malloc(4 * N);
    ev.e_ev = (float *)std::malloc(4 * N);
    ev.hist = (int32_t *)std::malloc(4 * N);
    if (!ev.x_um || !ev.y_um || !ev.z_um || !ev.e_ev || !ev.hist) {
        fd2_free_events(&ev);
        return FD2_ERR_OUT_OF_MEMORY;
    }
    if (n) {
        std::memcpy(ev.x_um, x.data(), 4 * n);
        std::memcpy(ev.y_um, y.data(), 4 * n);
        std::memcpy(ev.z_um, z.data(), 4 * n);
        std::memcpy(ev.e_ev, e.data(), 4 * n);
        std::memcpy(ev.hist, h.data(), 4 * n);
    }
    *out = ev;
    return FD2_OK;
}

std::string output_name(const fd2_params &p, const char *prefix)
{
    std::string s = prefix;
    for (int k = 0; k < 10; ++k) {
        std::string t(p.tag[k]);
        while (!t.empty() && (t.back() == ' ' || t.back() == '\t')) t.pop_back();
        s += t;
        s += (k < 9) ? "_" : ".dat";
    }
    return s;
}

// Fortran Fw.d / Iw: right-justified, asterisks when the value does not fit.
static void fortran_field(std::string &out, const char *txt, int w)
{
    const int len = (int)std::strlen(txt);
    if (len > w) {
        out.append((size_t)w, '*');
    } else {
        out.append((size_t)(w - len), ' ');
        out.append(txt);
    }
}

std::string format_prf(const uint64_t *image, int32_t xdim, int32_t ydim, const fd2_geometry &g, double num_hist)
{
    // pixel counts of the writer loops: int((ub - lb) / pixel) per axis; the
    // outer loop runs over the y pixel index with the x-derived bound and the
    // inner over x with the y-derived bound, as in the reference
    const int32_t nx = (int32_t)((g.ub_x - g.lb_x) / (double)g.pixel);
    const int32_t ny = (int32_t)((g.ub_y - g.lb_y) / (double)g.pixel);
    const double inv_n = 1.0 / num_hist;
    std::string out;
    out.reserve((size_t)(nx + 1) * (size_t)(ny + 1) * 14);
    char b[64];
    for (int32_t jj = 0; jj < nx; ++jj) {
        for (int32_t ii = 0; ii < ny; ++ii) {
            uint64_t c = 0;
            if (ii < xdim && jj < ydim) c = image[(int64_t)ii * ydim + jj];
            std::snprintf(b, sizeof b, "%.4f", (double)c * inv_n);
            out.push_back(' ');
            fortran_field(out, b, 12);
            out.push_back('\n');
        }
        out.push_back('\n');
    }
    return out;
}

std::string format_phs(const int32_t *bins, int32_t num_bins)
{
    std::string out;
    char b[32];
    for (int32_t k = 0; k < num_bins; ++k) {
        std::snprintf(b, sizeof b, "%d", bins[k]);
        out.push_back(' ');
        fortran_field(out, b, 8);
        out.push_back('\n');
    }
    return out;
}

// Create a new file (the reference opens with STATUS='NEW').
fd2_status write_new_file(const std::string &path, const std::string &data)
{
    const int fd = ::open(path.c_str(), O_WRONLY | O_CREAT | O_EXCL, 0644);
    if (fd < 0) return errno == EEXIST ? FD2_ERR_FILE_EXISTS : FD2_ERR_IO;
    size_t off = 0;
    while (off < data.size()) {
        const ssize_t w = ::write(fd, data.data() + off, data.size() - off);
        if (w <= 0) {
            ::close(fd);
            return FD2_ERR_IO;
        }
        off += (size_t)w;
    }
    return ::close(fd) == 0 ? FD2_OK : FD2_ERR_IO;
}

// ---- streaming EDE readers

namespace {

// One whitespace-delimited token of at most 63 characters as a real; a
// Fortran 'd' exponent is read as 'e' (parse_real's rule, without a copy to
// the heap).
bool token_real(const char *t, size_t len, double *out)
{
    char b[64];
    if (len == 0 || len >= sizeof b) return false;
    for (size_t k = 0; k < len; ++k) b[k] = (t[k] == 'd' || t[k] == 'D') ? 'e' : t[k];
    b[len] = '\0';
    char *end = nullptr;
    errno = 0;
    const double v = std::strtod(b, &end);
    if (end != b + len || errno == ERANGE) return false;
    *out = v;
    return true;
}

bool token_int(const char *t, size_t len, int32_t *out)
{
    char b[64];
    if (len == 0 || len >= sizeof b) return false;
    std::memcpy(b, t, len);
    b[len] = '\0';
    char *end = nullptr;
    errno = 0;
    const long v = std::strtol(b, &end, 10);
    if (end != b + len || errno == ERANGE || v < INT32_MIN || v > INT32_MAX) return false;
    *out = (int32_t)v;
    return true;
}

inline bool blank(char c) { return c == ' ' || c == '\t' || c == '\r' || c == '\v' || c == '\f'; }

// 1: an event row, 0: a comment or blank line, -1: a malformed row.  The
// first five tokens are read; more are ignored.
int parse_row(const char *s, double v[4], int32_t *hist)
{
    while (blank(*s)) ++s;
    if (*s == '#' || *s == '\0') return 0;
    const char *tok[5];
    size_t len[5];
    for (int k = 0; k < 5; ++k) {
        while (blank(*s)) ++s;
        if (*s == '\0') return -1;
        tok[k] = s;
        while (*s && !blank(*s)) ++s;
        len[k] = (size_t)(s - tok[k]);
    }
    for (int k = 0; k < 4; ++k)
        if (!token_real(tok[k], len[k], &v[k])) return -1;
    return token_int(tok[4], len[4], hist) ? 1 : -1;
}

}  // namespace

fd2_status stream_events_text(const char *path, int64_t batch, const TextSink &sink)
{
    if (!path || batch <= 0) return FD2_ERR_INVALID_ARGUMENT;
    FILE *f = std::fopen(path, "rb");
    if (!f) return FD2_ERR_IO;
    const size_t cap = (size_t)batch;
    std::vector<double> x(cap), y(cap), z(cap), e(cap);
    std::vector<int32_t> h(cap);
    size_t fill = 0;
    std::vector<char> buf((size_t)1 << 22);
    size_t have = 0;
    bool eof = false;
    fd2_status st = FD2_OK;
    auto row = [&](const char *line) {
        double v[4];
        int32_t hh = 0;
        const int r = parse_row(line, v, &hh);
        if (r < 0) return FD2_ERR_PARSE;
        if (r == 0) return FD2_OK;
        x[fill] = v[0];
        y[fill] = v[1];
        z[fill] = v[2];
        e[fill] = v[3];
        h[fill] = hh;
        if (++fill == cap) {
            fill = 0;
            return sink(x.data(), y.data(), z.data(), e.data(), h.data(), (int64_t)cap);
        }
        return FD2_OK;
    };
    while (st == FD2_OK) {
        if (!eof) {
            const size_t r = std::fread(buf.data() + have, 1, buf.size() - 1 - have, f);
            if (r == 0) {
                if (std::ferror(f)) st = FD2_ERR_IO;
                eof = true;
            }
            have += r;
        }
        size_t start = 0;
        while (st == FD2_OK) {
            char *nl = (char *)std::memchr(buf.data() + start, '\n', have - start);
            if (!nl) break;
            *nl = '\0';
            st = row(buf.data() + start);
            start = (size_t)(nl - buf.data()) + 1;
        }
        if (st != FD2_OK) break;
        if (eof) {
            if (start < have) {  // last row without a newline
                buf[have] = '\0';
                st = row(buf.data() + start);
            }
            break;
        }
        if (start == 0 && have == buf.size() - 1) {
            st = FD2_ERR_PARSE;  // a row longer than the read buffer
            break;
        }
        std::memmove(buf.data(), buf.data() + start, have - start);
        have -= start;
    }
    std::fclose(f);
    if (st == FD2_OK && fill > 0) st = sink(x.data(), y.data(), z.data(), e.data(), h.data(), (int64_t)fill);
    return st;
}

fd2_status stream_events_binary(const char *path, int64_t batch, const BinHeaderSink &on_header,
                                const BinSink &sink)
{
    if (!path || batch <= 0) return FD2_ERR_INVALID_ARGUMENT;
    FILE *f = std::fopen(path, "rb");
    if (!f) return FD2_ERR_IO;
    char magic[8];
    BinHeader hd{};
    bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, kBinMagic, 8) == 0 &&
              std::fread(&hd.n, 8, 1, f) == 1 && std::fread(&hd.num_hist, 4, 1, f) == 1 &&
              std::fread(&hd.has_geom, 4, 1, f) == 1 && hd.n >= 0 && hd.n < (int64_t)1 << 34;
    if (!ok) {
        std::fclose(f);
        return FD2_ERR_PARSE;
    }
    fd2_status st = on_header ? on_header(hd) : FD2_OK;
    const size_t cap = (size_t)std::min<int64_t>(batch, std::max<int64_t>(hd.n, 1));
    std::vector<float> plane[4];
    for (auto &v : plane) v.resize(cap);
    std::vector<int32_t> h(cap);
    std::vector<uint16_t> g(hd.has_geom ? cap : 0);
    const int64_t off0 = 24;  // magic, n, num_hist, has_geom
    for (int64_t i = 0; st == FD2_OK && i < hd.n; i += (int64_t)cap) {
        const size_t k = (size_t)std::min<int64_t>((int64_t)cap, hd.n - i);
        // planes x, y, z, e, hist (4 bytes each), then geometry ids (2 bytes)
        for (int p = 0; ok && p < 5; ++p) {
            void *dst = p < 4 ? (void *)plane[p].data() : (void *)h.data();
            ok = fseeko(f, (off_t)(off0 + (int64_t)p * hd.n * 4 + i * 4), SEEK_SET) == 0 &&
                 std::fread(dst, 4, k, f) == k;
        }
        if (ok && hd.has_geom)
            ok = fseeko(f, (off_t)(off0 + 5 * hd.n * 4 + i * 2), SEEK_SET) == 0 && std::fread(g.data(), 2, k, f) == k;
        if (!ok) {
            st = FD2_ERR_PARSE;
            break;
        }
        st = sink(plane[0].data(), plane[1].data(), plane[2].data(), plane[3].data(), h.data(),
                  hd.has_geom ? g.data() : nullptr, (int64_t)k);
    }
    std::fclose(f);
    return st;
}

}  // namespace fd2host
