// io.cpp -- sparse tensor files and host model initialisation.
//
// Replaces ImportSparseTensor / ExportSparseTensor (IntelLabs/ALTO
// src/sptensor.cpp:23-258) and KruskalModelRandomInit
// (src/kruskal_model.cpp:109-125).  The .tns reader keeps the reference's
// rules (lines of "i1 ... iN value"; lines that are empty or start with '#'
// are skipped; N = tokens - 1 on the first data line; dims = largest index
// seen; 1-based unless zero_based) but maps the file and parses it in
// parallel chunks split at line boundaries.
#include <fcntl.h>
#include <omp.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/altob.h"

namespace altob {
altob_status fail(altob_status s, const std::string& msg);
}
using altob::fail;

namespace {

struct Mapped {
    const char* p = nullptr;
    size_t n = 0;
    int fd = -1;
    ~Mapped()
    {
        if (p && n) munmap((void*)p, n);
        if (fd >= 0) close(fd);
    }
};

bool map_file(const char* path, Mapped& m)
{
    m.fd = open(path, O_RDONLY);
    if (m.fd < 0) return false;
    struct stat sb;
    if (fstat(m.fd, &sb) != 0) return false;
    m.n = (size_t)sb.st_size;
    if (m.n == 0) return true;
    void* p = mmap(nullptr, m.n, PROT_READ, MAP_PRIVATE, m.fd, 0);
    if (p == MAP_FAILED) {
        m.n = 0;
        return false;
    }
    madvise(p, m.n, MADV_SEQUENTIAL);
    m.p = (const char*)p;
    return true;
}

// A data line: more than just the newline and not a comment
// (sptensor.cpp:86, 115, 145: nread > 1 && line[0] != '#').
inline bool is_data(const char* s, const char* e, const char* end)
{
    size_t nread = (size_t)(e - s) + (e < end ? 1 : 0);
    return nread > 1 && s[0] != '#';
}

inline const char* line_end(const char* s, const char* end)
{
    const void* nl = memchr(s, '\n', (size_t)(end - s));
    return nl ? (const char*)nl : end;
}

// strtoull / strtod on a buffer that is not NUL terminated: copy the token.
inline const char* next_u64(const char* s, const char* e, unsigned long long* v)
{
    while (s < e && (*s == ' ' || *s == '\t')) ++s;
    unsigned long long x = 0;
    const char* t = s;
    while (t < e && *t >= '0' && *t <= '9') {
        x = x * 10 + (unsigned)(*t - '0');
        ++t;
    }
    *v = x;
    return t;
}

inline const char* next_f64(const char* s, const char* e, double* v)
{
    while (s < e && (*s == ' ' || *s == '\t')) ++s;
    char buf[64];
    size_t k = 0;
    while (s + k < e && k < sizeof(buf) - 1 && s[k] != ' ' && s[k] != '\t' && s[k] != '\r' && s[k] != '\n') {
        buf[k] = s[k];
        ++k;
    }
    buf[k] = 0;
    *v = strtod(buf, nullptr);
    return s + k;
}

altob_coo* new_coo(int nmode, uint64_t nnz)
{
    altob_coo* c = (altob_coo*)calloc(1, sizeof(altob_coo));
    if (!c) return nullptr;
    c->nmode = nmode;
    c->nnz = nnz;
    c->cidx = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)nmode * (nnz ? nnz : 1));
    c->vals = (double*)malloc(sizeof(double) * (nnz ? nnz : 1));
    if (!c->cidx || !c->vals) {
        free(c->cidx);
        free(c->vals);
        free(c);
        return nullptr;
    }
    return c;
}

}  // namespace

extern "C" {

altob_status altob_read_tns(const char* path, int zero_based, altob_coo** out)
{
    if (!path || !out) return fail(ALTOB_ERR_ARG, "NULL argument");
    *out = nullptr;
    Mapped m;
    if (!map_file(path, m)) return fail(ALTOB_ERR_IO, std::string("cannot open ") + path);
    const char* beg = m.p;
    const char* end = m.p + m.n;
    // number of modes from the first data line (sptensor.cpp:84-96)
    int nmode = -1;
    for (const char* s = beg; s < end;) {
        const char* e = line_end(s, end);
        if (is_data(s, e, end)) {
            int tokens = 0;
            const char* t = s;
            while (t < e) {
                while (t < e && (*t == ' ' || *t == '\t' || *t == '\r')) ++t;
                if (t >= e) break;
                ++tokens;
                while (t < e && *t != ' ' && *t != '\t' && *t != '\r') ++t;
            }
            nmode = tokens - 1;
            break;
        }
        s = e + 1;
    }
    if (nmode < 1 || nmode > ALTOB_MAX_MODES) return fail(ALTOB_ERR_IO, "bad or missing first data line");
    // chunks split at line starts
    int nth = std::max(1, omp_get_max_threads());
    size_t nchunk = std::max<size_t>(1, std::min<size_t>((size_t)nth * 4, m.n / 4096 + 1));
    std::vector<const char*> cs(nchunk + 1);
    cs[0] = beg;
    cs[nchunk] = end;
    for (size_t c = 1; c < nchunk; ++c) {
        const char* p = beg + (m.n * c) / nchunk;
        if (p < cs[c - 1]) p = cs[c - 1];
        if (p > beg && p < end && p[-1] != '\n') p = std::min(end, line_end(p, end) + 1);
        cs[c] = p;
    }
    std::vector<uint64_t> cnt(nchunk, 0);
#pragma omp parallel for schedule(dynamic, 1)
    for (long c = 0; c < (long)nchunk; ++c) {
        uint64_t k = 0;
        for (const char* s = cs[c]; s < cs[c + 1];) {
            const char* e = line_end(s, end);
            if (is_data(s, e, end)) ++k;
            s = e + 1;
        }
        cnt[c] = k;
    }
    std::vector<uint64_t> off(nchunk + 1, 0);
    for (size_t c = 0; c < nchunk; ++c) off[c + 1] = off[c] + cnt[c];
    const uint64_t nnz = off[nchunk];
    altob_coo* coo = new_coo(nmode, nnz);
    if (!coo) return fail(ALTOB_ERR_NOMEM, "host allocation failed");
    std::vector<std::vector<uint64_t>> dmax(nchunk, std::vector<uint64_t>(nmode, 0));
    const uint64_t one_based = zero_based ? 0 : 1;
    int bad = 0;
#pragma omp parallel for schedule(dynamic, 1) reduction(| : bad)
    for (long c = 0; c < (long)nchunk; ++c) {
        uint64_t k = off[c];
        for (const char* s = cs[c]; s < cs[c + 1];) {
            const char* e = line_end(s, end);
            if (is_data(s, e, end)) {
                const char* t = s;
                for (int n = 0; n < nmode; ++n) {
                    unsigned long long v;
                    t = next_u64(t, e, &v);
                    // dims: index + zero_based (sptensor.cpp:120-123); index: v - one_based
                    uint64_t dimv = v + (uint64_t)zero_based;
                    if (dimv > dmax[c][n]) dmax[c][n] = dimv;
                    if (v < one_based) bad = 1;
                    coo->cidx[(uint64_t)n * nnz + k] = v - one_based;
                }
                double x;
                next_f64(t, e, &x);
                coo->vals[k] = x;
                ++k;
            }
            s = e + 1;
        }
    }
    if (bad) {
        altob_coo_free(coo);
        return fail(ALTOB_ERR_IO, "index 0 in a 1-based .tns file");
    }
    for (int n = 0; n < nmode; ++n) {
        uint64_t d = 0;
        for (size_t c = 0; c < nchunk; ++c) d = std::max(d, dmax[c][n]);
        coo->dims[n] = d;
    }
    *out = coo;
    return ALTOB_OK;
}

altob_status altob_read_bin(const char* path, altob_coo** out)
{
    if (!path || !out) return fail(ALTOB_ERR_ARG, "NULL argument");
    *out = nullptr;
    FILE* f = fopen(path, "rb");
    if (!f) return fail(ALTOB_ERR_IO, std::string("cannot open ") + path);
    uint64_t nm = 0, nnz = 0;
    uint64_t dims[ALTOB_MAX_MODES] = {0};
    bool ok = fread(&nm, 8, 1, f) == 1;
    // the reference writes an int into this 8-byte field (sptensor.cpp:59):
    // only the low 32 bits are meaningful
    nm &= 0xffffffffull;
    ok = ok && nm >= 1 && nm <= ALTOB_MAX_MODES;
    ok = ok && fread(dims, 8, nm, f) == nm;
    ok = ok && fread(&nnz, 8, 1, f) == 1;
    if (!ok) {
        fclose(f);
        return fail(ALTOB_ERR_IO, "bad binary tensor header");
    }
    altob_coo* coo = new_coo((int)nm, nnz);
    if (!coo) {
        fclose(f);
        return fail(ALTOB_ERR_NOMEM, "host allocation failed");
    }
    for (uint64_t n = 0; n < nm; ++n) coo->dims[n] = dims[n];
    ok = fread(coo->cidx, 8, nm * nnz, f) == nm * nnz;
    ok = ok && fread(coo->vals, 8, nnz, f) == nnz;
    fclose(f);
    if (!ok) {
        altob_coo_free(coo);
        return fail(ALTOB_ERR_IO, "truncated binary tensor");
    }
    *out = coo;
    return ALTOB_OK;
}

altob_status altob_write_bin(const char* path, const altob_coo* c)
{
    if (!path || !c) return fail(ALTOB_ERR_ARG, "NULL argument");
    FILE* f = fopen(path, "wb");
    if (!f) return fail(ALTOB_ERR_IO, std::string("cannot create ") + path);
    uint64_t nm = (uint64_t)c->nmode;
    bool ok = fwrite(&nm, 8, 1, f) == 1;
    ok = ok && fwrite(c->dims, 8, nm, f) == nm;
    ok = ok && fwrite(&c->nnz, 8, 1, f) == 1;
    ok = ok && fwrite(c->cidx, 8, nm * c->nnz, f) == nm * c->nnz;
    ok = ok && fwrite(c->vals, 8, c->nnz, f) == c->nnz;
    ok = (fclose(f) == 0) && ok;
    return ok ? ALTOB_OK : fail(ALTOB_ERR_IO, "write failed");
}

altob_status altob_write_tns(const char* path, const altob_coo* c)
{
    if (!path || !c) return fail(ALTOB_ERR_ARG, "NULL argument");
    FILE* f = fopen(path, "w");
    if (!f) return fail(ALTOB_ERR_IO, std::string("cannot create ") + path);
    for (uint64_t i = 0; i < c->nnz; ++i) {
        for (int n = 0; n < c->nmode; ++n) fprintf(f, "%llu ", (unsigned long long)(c->cidx[(uint64_t)n * c->nnz + i] + 1));
        fprintf(f, "%g\n", c->vals[i]);
    }
    return fclose(f) == 0 ? ALTOB_OK : fail(ALTOB_ERR_IO, "write failed");
}

void altob_coo_free(altob_coo* c)
{
    if (!c) return;
    free(c->cidx);
    free(c->vals);
    free(c);
}

altob_status altob_kruskal_random_init(int nmode, const uint64_t* dims, uint64_t rank, unsigned seed,
                                       altob_dtype ftype, void* const* h_factors, void* h_lambda)
{
    if (!dims || !h_factors || nmode < 1 || nmode > ALTOB_MAX_MODES || rank < 1)
        return fail(ALTOB_ERR_ARG, "bad argument");
    if (ftype != ALTOB_F64 && ftype != ALTOB_F32) return fail(ALTOB_ERR_ARG, "dtype must be F64 or F32");
    for (uint64_t r = 0; r < rank && h_lambda; ++r) {
        if (ftype == ALTOB_F64) ((double*)h_lambda)[r] = 1.0;
        else ((float*)h_lambda)[r] = 1.0f;
    }
    srand(seed);
    for (int n = 0; n < nmode; ++n) {
        if (!h_factors[n]) return fail(ALTOB_ERR_ARG, "a factor pointer is NULL");
        const uint64_t cnt = dims[n] * rank;
        for (uint64_t i = 0; i < cnt; ++i) {
            // (FType) rand() / RAND_MAX, evaluated in FType as the reference does
            if (ftype == ALTOB_F64) ((double*)h_factors[n])[i] = (double)rand() / RAND_MAX;
            else ((float*)h_factors[n])[i] = (float)rand() / RAND_MAX;
        }
    }
    return ALTOB_OK;
}

}  // extern "C"
