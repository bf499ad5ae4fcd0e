/*
 * gf_textout.cpp -- the catalog writers: galfast's os_textout output module
 * (src/pipeline.cpp:199-289) and os_fitsout (pipeline.cpp:767-1035) over host
 * tables of this library.
 *
 * The file is the reference's: a header line "# " followed by the definition of
 * every output column and a space (otable::serialize_header,
 * src/common/otable.cpp:542-558; columndef::serialize_def, :409-467), an
 * optional "# generated with galfast version ..." line, then one line per
 * visible row (hidden rows are skipped, mask_output, pipeline.cpp:221-233) with
 * every column's components printed with the column's printf format and
 * separated by one space (otable::serialize_body, otable.cpp:562-584; fmtout,
 * src/common/otable.h:39-90).  Column order and formats follow the built-in
 * schema of otable::init (otable.cpp:719-745) and getSortedColumnsForOutput
 * (otable.cpp:517-540); the photometry and photometric-error columns are named
 * as os_photometry and os_photometricErrors name them
 * (photometry_host.cpp:87-122, photometricErrors_host.cpp:150-185).
 *
 * Formatting is this library's: numbers are converted with an exact
 * fixed-point routine (the correctly rounded decimal of the binary value,
 * ties to even, as glibc's printf), rows are formatted in parallel pieces on
 * host threads and written in order.
 *
 * The FITS catalog has os_fitsout's layout, written from the FITS standard (no
 * CFITSIO): an empty primary HDU, a binary table CATALOG with one column per
 * output column (TTYPE its primary name, TFORM its width and type code: D
 * double, E float, J int) and one big-endian row per visible row, then a binary
 * table METADATA with one row whose string column HEADER holds the column
 * definitions of the text header.
 */
#include "../../include/galfast_b200.h"
#include "gf_launch.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <condition_variable>
#include <cstddef>
#include <cstdio>
#include <cstring>
#include <functional>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

namespace {

/* ---------------- number formatting ---------------- */

/* printf("%[ ]W.Pf", v) for 0 <= P <= 9: the exact decimal of v rounded to P
 * digits, ties to even.  Returns the characters written to dst (no NUL; at
 * most 330 characters). */
int fmt_fixed(char *dst, double v, int prec, int width, bool space)
{
    char tmp[64];
    int n = 0;
    const bool neg = std::signbit(v);
    if (std::isnan(v) || std::isinf(v)) {
        if (neg) tmp[n++] = '-';
        else if (space) tmp[n++] = ' ';
        const char *w = std::isnan(v) ? "nan" : "inf";
        for (int i = 0; i < 3; i++) tmp[n++] = w[i];
    } else {
        static const uint64_t P10[10] = {1ull, 10ull, 100ull, 1000ull, 10000ull, 100000ull, 1000000ull, 10000000ull,
                                         100000000ull, 1000000000ull};
        const double a = std::fabs(v);
        unsigned __int128 N = 0;
        if (a != 0.0) {
            int e2 = 0;
            const double fr = std::frexp(a, &e2);                 /* a = fr 2^e2, fr in [0.5, 1) */
            const uint64_t m = (uint64_t)std::ldexp(fr, 53);      /* exact: 53 significant bits */
            const int e = e2 - 53;                                /* a = m 2^e */
            const unsigned __int128 prod = (unsigned __int128)m * P10[prec];
            if (e >= 0) {
                if (e > 40) {
                    /* beyond 2^93: printf itself */
                    char big[400];
                    const int k = std::snprintf(big, sizeof(big), space ? "% *.*f" : "%*.*f", width, prec, v);
                    memcpy(dst, big, (size_t)k);
                    return k;
                }
                N = prod << e;
            } else {
                const int s = -e;
                if (s < 120) {
                    unsigned __int128 q = prod >> s;
                    const unsigned __int128 r = prod - (q << s);
                    const unsigned __int128 half = (unsigned __int128)1 << (s - 1);
                    if (r > half || (r == half && (q & 1))) q++;
                    N = q;
                }
            }
        }
        unsigned __int128 ip = N / P10[prec];
        uint64_t fp = (uint64_t)(N % P10[prec]);
        if (neg) tmp[n++] = '-';
        else if (space) tmp[n++] = ' ';
        char digs[48];
        int nd = 0;
        do { digs[nd++] = (char)('0' + (int)(ip % 10)); ip /= 10; } while (ip);
        while (nd) tmp[n++] = digs[--nd];
        if (prec > 0) {
            tmp[n++] = '.';
            for (int i = prec - 1; i >= 0; i--) { tmp[n + i] = (char)('0' + (int)(fp % 10)); fp /= 10; }
            n += prec;
        }
    }
    int pad = width > n ? width - n : 0;
    for (int i = 0; i < pad; i++) dst[i] = ' ';
    memcpy(dst + pad, tmp, n);
    return pad + n;
}

/* printf("%[ ]Wd", v) */
int fmt_int(char *dst, int32_t v, int width, bool space)
{
    char tmp[24];
    int n = 0;
    int64_t x = v;
    if (x < 0) { tmp[n++] = '-'; x = -x; }
    else if (space) tmp[n++] = ' ';
    char digs[16];
    int nd = 0;
    do { digs[nd++] = (char)('0' + (int)(x % 10)); x /= 10; } while (x);
    while (nd) tmp[n++] = digs[--nd];
    int pad = width > n ? width - n : 0;
    for (int i = 0; i < pad; i++) dst[i] = ' ';
    memcpy(dst + pad, tmp, n);
    return pad + n;
}

/* ---------------- a shared pool of formatting threads ---------------- */
class FmtPool {
public:
    static FmtPool &get()
    {
        static FmtPool p;
        return p;
    }
    /* f(i) for i in [0, n) on the calling thread and up to threads - 1 workers */
    void run(int n, int threads, const std::function<void(int)> &f)
    {
        if (threads <= 1 || n <= 1) { for (int i = 0; i < n; i++) f(i); return; }
        std::lock_guard<std::mutex> one(run_mu_);           /* one parallel loop at a time */
        ensure(threads - 1);
        auto job = std::make_shared<Job>();
        job->f = &f;
        job->n = n;
        {
            std::lock_guard<std::mutex> g(mu_);
            cur_ = job;
            gen_++;
        }
        cv_.notify_all();
        work(*job);
        std::unique_lock<std::mutex> g(mu_);
        done_.wait(g, [&] { return job->done.load() >= n; });
    }
    ~FmtPool()
    {
        {
            std::lock_guard<std::mutex> g(mu_);
            stop_ = true;
            gen_++;
        }
        cv_.notify_all();
        for (auto &t : th_) t.join();
    }

private:
    struct Job {
        const std::function<void(int)> *f = nullptr;
        int n = 0;
        std::atomic<int> next{0}, done{0};
    };
    void ensure(int workers)
    {
        while ((int)th_.size() < workers) {
            uint64_t g0;
            {
                std::lock_guard<std::mutex> g(mu_);
                g0 = gen_;
            }
            th_.emplace_back([this, g0] { loop(g0); });
        }
    }
    void work(Job &j)
    {
        for (;;) {
            const int i = j.next.fetch_add(1);
            if (i >= j.n) break;
            (*j.f)(i);
            if (j.done.fetch_add(1) + 1 == j.n) {
                std::lock_guard<std::mutex> g(mu_);
                done_.notify_all();
            }
        }
    }
    void loop(uint64_t seen)
    {
        for (;;) {
            std::shared_ptr<Job> j;
            {
                std::unique_lock<std::mutex> g(mu_);
                cv_.wait(g, [&] { return stop_ || gen_ != seen; });
                if (stop_) return;
                seen = gen_;
                j = cur_;
            }
            if (j) work(*j);
        }
    }
    std::mutex run_mu_, mu_;
    std::condition_variable cv_, done_;
    std::vector<std::thread> th_;
    std::shared_ptr<Job> cur_;
    uint64_t gen_ = 0;
    bool stop_ = false;
};

/* ---------------- the output columns ---------------- */
enum Kind { F64, F32, I32 };

struct Field {
    Kind kind;
    size_t col_off;        /* offset of the column pointer inside gf_table */
    int ncomp;             /* components (vector columns: component-major, pitch = capacity) */
    int prec, width;
    bool space, comp_map;
};

struct ColumnDef {
    std::string def;       /* its part of the header line */
    Field f;
};

#define GF_OFF(m) offsetof(gf_table, m)

}  // namespace

struct gf_textout {
    FILE *fp = nullptr;
    std::vector<Field> fields;
    std::vector<int32_t> comp_ids;
    int threads = 1;
    int64_t rows = 0;
    int64_t bytes = 0;
    bool failed = false;
    std::mutex mu;          /* one write at a time */
    /* FITS catalogs (gf_fitsout_open) */
    bool fits = false;
    int64_t row_bytes = 0;          /* NAXIS1 of the CATALOG table */
    long naxis2_at = 0;             /* file offset of its NAXIS2 card */
    int64_t data_bytes = 0;         /* bytes of table rows written */
    std::string header_def;         /* the column definitions (METADATA extension) */
};

namespace {

/* Columns in the order of getSortedColumnsForOutput: the ranked built-in fields,
 * then the others sorted by name without regard to case. */
std::vector<ColumnDef> output_columns(const gf_textout_config &c)
{
    std::vector<ColumnDef> ranked, others;
    auto astro = [](size_t off) { return Field{F64, off, 2, 8, 13, true, false}; };
    ranked.push_back({"lb[2]", astro(GF_OFF(lb))});
    if (c.radec) ranked.push_back({"radec[2]", astro(GF_OFF(radec))});
    ranked.push_back({"XYZ[3]", Field{F32, GF_OFF(XYZ), 3, 2, 10, true, false}});
    ranked.push_back({"DM", Field{F32, GF_OFF(DM), 1, 3, 7, true, false}});
    {
        /* "abs" + band, with the aliases absmag and M1 and the band property
         * (os_skygen.cpp:851-857); serialize_def lists aliases in the table's
         * (byte-wise) name order, then the properties */
        const std::string band = c.band ? c.band : "";
        const std::string name = c.absband ? c.absband : ("abs" + band);
        /* unresolved multiples drop the M1 alias (it names the primary of absmag + "Sys",
         * unresolvedMultiples_host.cpp:56-80) */
        std::vector<std::string> alias = {"absmag"};
        if (!c.multiples) alias.push_back("M1");
        std::sort(alias.begin(), alias.end());
        std::string d = name + "{";
        for (auto &a : alias) d += "alias=" + a + ";";
        if (!band.empty()) d += "band=" + band + ";";
        d += "}";
        ranked.push_back({d, Field{F32, GF_OFF(absmag), 1, 3, 7, true, false}});
        if (c.multiples) {
            const std::string bp = band.empty() ? "" : "band=" + band + ";";
            others.push_back({name + "Sys[2]{class=magnitude;fieldNames=0:M1,1:M2;alias=absmagSys;" + bp + "}",
                              Field{F32, GF_OFF(absmagSys), 2, 3, 7, true, false}});
            others.push_back({name + "SysNcomp{type=int;fmt=%1d;}", Field{I32, GF_OFF(absmagSysNcomp), 1, 0, 1, false, false}});
        }
    }
    ranked.push_back({"comp", Field{I32, GF_OFF(comp), 1, 0, 3, false, true}});
    if (c.feh) ranked.push_back({"FeH", Field{F32, GF_OFF(FeH), 1, 3, 6, true, false}});
    /* provided as "FeH_comp{type=int; fmt=%3d;}" (GaussianFeH_host.cpp:46-47) */
    if (c.feh_comp) ranked.push_back({"FeH_comp{type=int;fmt=%3d;}", Field{I32, GF_OFF(FeH_comp), 1, 0, 3, false, false}});
    if (c.vcyl) ranked.push_back({"vcyl[3]", Field{F32, GF_OFF(vcyl), 3, 1, 7, true, false}});
    if (c.pm_coordsys == 0) ranked.push_back({"pmlb[3]", Field{F32, GF_OFF(pm), 3, 2, 8, true, false}});
    if (c.pm_coordsys == 1) ranked.push_back({"pmradec[3]", Field{F32, GF_OFF(pm), 3, 2, 8, true, false}});
    ranked.push_back({"Am", Field{F32, GF_OFF(Am), 1, 3, 6, false, false}});
    ranked.push_back({"AmInf", Field{F32, GF_OFF(AmInf), 1, 3, 6, false, false}});
    if (c.bandset && c.nbands > 0) {
        const std::string bs = c.bandset;
        std::string fn, ofn;
        for (int b = 0; b < c.nbands; b++) {
            const std::string bn = c.bands && c.bands[b] ? c.bands[b] : ("b" + std::to_string(b));
            if (b) { fn += ","; ofn += ","; }
            fn += std::to_string(b) + ":" + bn;
            ofn += std::to_string(b) + ":obs" + bn;
        }
        const std::string n = std::to_string(c.nbands);
        others.push_back({bs + "[" + n + "]{class=magnitude;fieldNames=" + fn + ";}",
                          Field{F32, GF_OFF(mags), c.nbands, 3, 7, true, false}});
        others.push_back({bs + "PhotoFlags{class=flags;}", Field{I32, GF_OFF(photoflags), 1, 0, 4, true, false}});
        if (c.photoerrors)
            others.push_back({"obs" + bs + "[" + n + "]{class=magnitude;fieldNames=" + ofn + ";}",
                              Field{F32, GF_OFF(obsmags), c.nbands, 3, 7, true, false}});
    }
    auto key = [](const std::string &d) {
        std::string k = d.substr(0, d.find_first_of("[{"));
        for (auto &ch : k) ch = (char)tolower((unsigned char)ch);
        return k;
    };
    std::stable_sort(others.begin(), others.end(), [&](const ColumnDef &a, const ColumnDef &b) { return key(a.def) < key(b.def); });
    ranked.insert(ranked.end(), others.begin(), others.end());
    return ranked;
}

template <typename T>
const T *col_ptr(const gf_table &t, size_t off)
{
    const T *p = nullptr;
    memcpy(&p, (const char *)&t + off, sizeof(p));
    return p;
}

/* the rows [r0, r1) of t that are not hidden, as text */
void format_rows(const gf_textout &w, const gf_table &t, int64_t r0, int64_t r1, std::string &out, int64_t &nrows)
{
    const size_t P = (size_t)t.capacity;
    const int32_t *hidden = t.hidden;
    static thread_local std::vector<char> linebuf(32768);
    char *line = linebuf.data();
    nrows = 0;
    for (int64_t r = r0; r < r1; r++) {
        if (hidden && hidden[r]) continue;
        int n = 0;
        for (const Field &f : w.fields) {
            for (int k = 0; k < f.ncomp; k++) {
                if (n) line[n++] = ' ';
                const size_t idx = (size_t)k * P + (size_t)r;
                if (f.kind == F64) {
                    n += fmt_fixed(line + n, col_ptr<double>(t, f.col_off)[idx], f.prec, f.width, f.space);
                } else if (f.kind == F32) {
                    n += fmt_fixed(line + n, (double)col_ptr<float>(t, f.col_off)[idx], f.prec, f.width, f.space);
                } else {
                    int32_t v = col_ptr<int32_t>(t, f.col_off)[idx];
                    if (f.comp_map && v >= 0 && v < (int32_t)w.comp_ids.size()) v = w.comp_ids[v];
                    n += fmt_int(line + n, v, f.width, f.space);
                }
            }
        }
        line[n++] = '\n';
        out.append(line, (size_t)n);
        nrows++;
    }
}

gf_status tfail(gf_status s, const std::string &m)
{
    gfk::set_last_error(m);
    return s;
}

/* ---------------- FITS (os_fitsout, src/pipeline.cpp:767-1035) ---------------- */

/* One 80-character header card (FITS standard 4.0, section 4.1): the keyword in
 * columns 1-8, "= " in 9-10, then a fixed-format value: integers and logicals
 * right-justified to column 30, strings quoted from column 11 and padded to at
 * least 8 characters inside the quotes. */
std::string fits_card(const std::string &key, const std::string &value, bool quoted)
{
    std::string c = key;
    c.resize(8, ' ');
    if (key != "END") {
        c += "= ";
        if (quoted) {
            std::string v;
            for (char ch : value) { v += ch; if (ch == '\'') v += '\''; }
            if (v.size() < 8) v.resize(8, ' ');
            c += "'" + v + "'";
        } else {
            std::string v = value;
            if (v.size() < 20) v = std::string(20 - v.size(), ' ') + v;
            c += v;
        }
    }
    c.resize(80, ' ');
    return c;
}

std::string fits_pad(std::string h)
{
    h.resize((h.size() + 2879) / 2880 * 2880, ' ');
    return h;
}

char fits_code(Kind k) { return k == F64 ? 'D' : k == F32 ? 'E' : 'J'; }
size_t kind_bytes(Kind k) { return k == F64 ? 8 : 4; }

/* the primary name of a column (its definition up to "[" or "{") */
std::string primary_name(const std::string &def) { return def.substr(0, def.find_first_of("[{")); }

inline void put_be32(unsigned char *d, uint32_t v)
{
    d[0] = (unsigned char)(v >> 24); d[1] = (unsigned char)(v >> 16); d[2] = (unsigned char)(v >> 8); d[3] = (unsigned char)v;
}
inline void put_be64(unsigned char *d, uint64_t v)
{
    put_be32(d, (uint32_t)(v >> 32));
    put_be32(d + 4, (uint32_t)v);
}

/* the rows [r0, r1) of t that are not hidden, as big-endian FITS table rows */
void pack_rows(const gf_textout &w, const gf_table &t, int64_t r0, int64_t r1, std::string &out, int64_t &nrows)
{
    const size_t P = (size_t)t.capacity;
    const int32_t *hidden = t.hidden;
    std::vector<unsigned char> row((size_t)w.row_bytes);
    nrows = 0;
    for (int64_t r = r0; r < r1; r++) {
        if (hidden && hidden[r]) continue;
        unsigned char *d = row.data();
        for (const Field &f : w.fields) {
            for (int k = 0; k < f.ncomp; k++) {
                const size_t idx = (size_t)k * P + (size_t)r;
                if (f.kind == F64) {
                    uint64_t b;
                    memcpy(&b, &col_ptr<double>(t, f.col_off)[idx], 8);
                    put_be64(d, b);
                    d += 8;
                } else if (f.kind == F32) {
                    uint32_t b;
                    memcpy(&b, &col_ptr<float>(t, f.col_off)[idx], 4);
                    put_be32(d, b);
                    d += 4;
                } else {
                    int32_t v = col_ptr<int32_t>(t, f.col_off)[idx];
                    if (f.comp_map && v >= 0 && v < (int32_t)w.comp_ids.size()) v = w.comp_ids[v];
                    put_be32(d, (uint32_t)v);
                    d += 4;
                }
            }
        }
        out.append((const char *)row.data(), row.size());
        nrows++;
    }
}

/* the header of a binary-table extension; *naxis2_at receives the offset of the
 * NAXIS2 card within it */
std::string bintable_header(int64_t naxis1, int64_t naxis2, const std::vector<std::pair<std::string, std::string>> &cols,
                            const std::string &extname, size_t *naxis2_at)
{
    std::string h;
    h += fits_card("XTENSION", "BINTABLE", true);
    h += fits_card("BITPIX", "8", false);
    h += fits_card("NAXIS", "2", false);
    h += fits_card("NAXIS1", std::to_string(naxis1), false);
    if (naxis2_at) *naxis2_at = h.size();
    h += fits_card("NAXIS2", std::to_string(naxis2), false);
    h += fits_card("PCOUNT", "0", false);
    h += fits_card("GCOUNT", "1", false);
    h += fits_card("TFIELDS", std::to_string(cols.size()), false);
    for (size_t i = 0; i < cols.size(); i++) {
        h += fits_card("TTYPE" + std::to_string(i + 1), cols[i].first, true);
        h += fits_card("TFORM" + std::to_string(i + 1), cols[i].second, true);
    }
    h += fits_card("EXTNAME", extname, true);
    h += fits_card("END", "", false);
    return fits_pad(h);
}

bool put(gf_textout *w, const std::string &b)
{
    if (fwrite(b.data(), 1, b.size(), w->fp) != b.size()) return false;
    w->bytes += (int64_t)b.size();
    return true;
}

/* close a FITS catalog: pad the CATALOG rows to a whole record, write the row
 * count into its header, and append the METADATA extension (one row, one
 * string column HEADER holding the column definitions, as os_fitsout's
 * destructor writes it) */
bool fits_finish(gf_textout *w)
{
    const int64_t pad = (2880 - w->data_bytes % 2880) % 2880;
    if (!put(w, std::string((size_t)pad, '\0'))) return false;
    const long end = ftell(w->fp);
    if (fseek(w->fp, w->naxis2_at, SEEK_SET) != 0) return false;
    const std::string c = fits_card("NAXIS2", std::to_string(w->rows), false);
    if (fwrite(c.data(), 1, c.size(), w->fp) != c.size()) return false;
    if (fseek(w->fp, end, SEEK_SET) != 0) return false;
    const std::string &hd = w->header_def;
    const int64_t len = std::max<int64_t>((int64_t)hd.size(), 1);
    if (!put(w, bintable_header(len, 1, {{"HEADER", std::to_string(len) + "A"}}, "METADATA", nullptr))) return false;
    std::string data = hd;
    data.resize((size_t)len, '\0');
    data.resize(((size_t)len + 2879) / 2880 * 2880, '\0');
    return put(w, data);
}

}  // namespace

extern "C" {

gf_status gf_fitsout_open(const char *path, const gf_textout_config *cfg, gf_textout **out)
{
    if (!path || !cfg || !out) return tfail(GF_E_INVALID, "invalid FITS output arguments");
    if (cfg->nbands < 0 || cfg->nbands > GF_MAX_BANDS) return tfail(GF_E_INVALID, "band count out of range");
    if (cfg->pm_coordsys < -1 || cfg->pm_coordsys > 1) return tfail(GF_E_INVALID, "pm_coordsys must be -1, 0 or 1");
    gf_textout *w = new gf_textout();
    w->fits = true;
    w->fp = fopen(path, "w+b");
    if (!w->fp) {
        delete w;
        return tfail(GF_E_INVALID, std::string("cannot open ") + path);
    }
    setvbuf(w->fp, nullptr, _IOFBF, (size_t)8 << 20);
    std::vector<std::pair<std::string, std::string>> cols;
    for (auto &c : output_columns(*cfg)) {
        w->header_def += c.def + " ";
        w->fields.push_back(c.f);
        cols.push_back({primary_name(c.def), std::to_string(c.f.ncomp) + fits_code(c.f.kind)});
        w->row_bytes += (int64_t)c.f.ncomp * (int64_t)kind_bytes(c.f.kind);
    }
    if (cfg->version && cfg->version[0]) w->header_def += std::string("\n# generated with galfast version ") + cfg->version;
    if (cfg->comp_ids && cfg->ncomp > 0) w->comp_ids.assign(cfg->comp_ids, cfg->comp_ids + cfg->ncomp);
    w->threads = cfg->threads > 0 ? cfg->threads : (int)std::max(1u, std::thread::hardware_concurrency());
    /* an empty primary HDU, then the CATALOG table (its row count written at close) */
    std::string primary = fits_card("SIMPLE", "T", false) + fits_card("BITPIX", "8", false) + fits_card("NAXIS", "0", false) +
                          fits_card("EXTEND", "T", false) + fits_card("END", "", false);
    size_t at = 0;
    const std::string cat = bintable_header(w->row_bytes, 0, cols, "CATALOG", &at);
    primary = fits_pad(primary);
    w->naxis2_at = (long)(primary.size() + at);
    if (!put(w, primary) || !put(w, cat)) {
        fclose(w->fp);
        delete w;
        return tfail(GF_E_INVALID, "cannot write the FITS headers");
    }
    *out = w;
    return GF_OK;
}

gf_status gf_textout_open(const char *path, const gf_textout_config *cfg, gf_textout **out)
{
    if (!path || !cfg || !out) return tfail(GF_E_INVALID, "invalid text output arguments");
    if (cfg->nbands < 0 || cfg->nbands > GF_MAX_BANDS) return tfail(GF_E_INVALID, "band count out of range");
    if (cfg->pm_coordsys < -1 || cfg->pm_coordsys > 1) return tfail(GF_E_INVALID, "pm_coordsys must be -1, 0 or 1");
    gf_textout *w = new gf_textout();
    w->fp = fopen(path, "wb");
    if (!w->fp) {
        delete w;
        return tfail(GF_E_INVALID, std::string("cannot open ") + path);
    }
    setvbuf(w->fp, nullptr, _IOFBF, (size_t)8 << 20);
    std::string h = "# ";
    for (auto &c : output_columns(*cfg)) {
        h += c.def + " ";
        w->fields.push_back(c.f);
    }
    if (cfg->version && cfg->version[0]) h += std::string("\n# generated with galfast version ") + cfg->version;
    h += "\n";
    if (cfg->comp_ids && cfg->ncomp > 0) w->comp_ids.assign(cfg->comp_ids, cfg->comp_ids + cfg->ncomp);
    w->threads = cfg->threads > 0 ? cfg->threads : (int)std::max(1u, std::thread::hardware_concurrency());
    if (fwrite(h.data(), 1, h.size(), w->fp) != h.size()) {
        fclose(w->fp);
        delete w;
        return tfail(GF_E_INVALID, "cannot write the text header");
    }
    w->bytes = (int64_t)h.size();
    *out = w;
    return GF_OK;
}

gf_status gf_textout_write(gf_textout *w, const gf_table *host, int64_t begin, int64_t end)
{
    if (!w || !host) return tfail(GF_E_INVALID, "invalid text output arguments");
    if (begin < 0 || end < begin || end > host->capacity) return tfail(GF_E_INVALID, "invalid row range");
    for (const Field &f : w->fields) {
        const void *p = nullptr;
        memcpy(&p, (const char *)host + f.col_off, sizeof(p));
        if (!p) return tfail(GF_E_INVALID, "the host table lacks a column of the text output");
        if ((f.col_off == GF_OFF(mags) || f.col_off == GF_OFF(obsmags)) && host->nbands < f.ncomp)
            return tfail(GF_E_INVALID, "the host table has fewer bands than the text output");
    }
    std::lock_guard<std::mutex> g(w->mu);
    if (w->failed) return tfail(GF_E_STATE, "an earlier write failed");
    const int64_t n = end - begin;
    const int64_t piece = 16384;
    const int npieces = (int)((n + piece - 1) / piece);
    std::vector<std::string> buf(npieces);
    std::vector<int64_t> cnt(npieces, 0);
    FmtPool::get().run(npieces, w->threads, [&](int i) {
        const int64_t a = begin + (int64_t)i * piece, b = std::min(end, a + piece);
        if (w->fits) {
            buf[i].reserve((size_t)(b - a) * (size_t)w->row_bytes);
            pack_rows(*w, *host, a, b, buf[i], cnt[i]);
        } else {
            buf[i].reserve((size_t)(b - a) * 256);
            format_rows(*w, *host, a, b, buf[i], cnt[i]);
        }
    });
    for (int i = 0; i < npieces; i++) {
        if (fwrite(buf[i].data(), 1, buf[i].size(), w->fp) != buf[i].size()) {
            w->failed = true;
            return tfail(GF_E_INVALID, "write error");
        }
        w->rows += cnt[i];
        w->bytes += (int64_t)buf[i].size();
        w->data_bytes += (int64_t)buf[i].size();
    }
    return GF_OK;
}

int gf_textout_multi_sink(void *set, int32_t model, const gf_table *host, const int64_t *row_begin, const int64_t *row_count)
{
    (void)model;
    const gf_textout_set *s = (const gf_textout_set *)set;
    if (!s || !host) return 1;
    for (int32_t j = 0; j < s->njobs; j++) {
        if (!s->writers[j] || row_count[j] <= 0) continue;
        if (gf_textout_write(s->writers[j], host, row_begin[j], row_begin[j] + row_count[j]) != GF_OK) return 1;
    }
    return 0;
}

gf_status gf_textout_close(gf_textout *w, int64_t *rows, int64_t *bytes)
{
    if (!w) return GF_OK;
    gf_status st = w->failed ? GF_E_INVALID : GF_OK;
    if (w->fits && w->fp && st == GF_OK && !fits_finish(w)) st = tfail(GF_E_INVALID, "cannot finish the FITS file");
    if (w->fp && fclose(w->fp) != 0) st = tfail(GF_E_INVALID, "close error");
    if (rows) *rows = w->rows;
    if (bytes) *bytes = w->bytes;
    delete w;
    return st;
}

}  /* extern "C" */
