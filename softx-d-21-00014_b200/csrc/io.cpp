// Files: XAMG's binary system format (src/io/detail/reader.inl:47-177) and
// the library's own multigrid hierarchy files.
#include "io.h"

#include <cstdio>
#include <cstring>
#include <memory>

namespace xg {

namespace {

struct File {
    FILE *f = nullptr;
    File(const char *path, const char *mode) : f(std::fopen(path, mode)) {}
    ~File() {
        if (f) std::fclose(f);
    }
};

void read_exact(FILE *f, void *p, size_t bytes, const char *what) {
    if (bytes && std::fread(p, 1, bytes, f) != bytes)
        throw Error(XAMG_ERR_INVALID_ARG, std::string("file ends inside ") + what);
}

void write_exact(FILE *f, const void *p, size_t bytes) {
    if (bytes && std::fwrite(p, 1, bytes, f) != bytes)
        throw Error(XAMG_ERR_INTERNAL, "write failed");
}

uint64_t file_size(FILE *f) {
    const long cur = std::ftell(f);
    std::fseek(f, 0, SEEK_END);
    const long end = std::ftell(f);
    std::fseek(f, cur, SEEK_SET);
    return end < 0 ? 0 : (uint64_t)end;
}

// FNV-1a over a byte range, continuing from h.
uint64_t fnv1a(uint64_t h, const void *p, size_t bytes) {
    const unsigned char *c = (const unsigned char *)p;
    for (size_t i = 0; i < bytes; ++i) {
        h ^= c[i];
        h *= 1099511628211ull;
    }
    return h;
}

const char MAGIC[8] = {'X', 'A', 'M', 'G', 'B', '2', 'H', 'I'};
const uint32_t VERSION = 1;

void write_csr(FILE *f, const HCsr &m) {
    const uint64_t h[3] = {m.nrows, m.ncols, (uint64_t)m.col.size()};
    write_exact(f, h, sizeof(h));
    write_exact(f, m.row.data(), m.row.size() * 4);
    write_exact(f, m.col.data(), m.col.size() * 4);
    write_exact(f, m.val.data(), m.val.size() * 8);
}

HCsr read_csr(FILE *f) {
    uint64_t h[3];
    read_exact(f, h, sizeof(h), "a hierarchy matrix header");
    XG_REQUIRE(h[0] < (1ull << 32) && h[1] < (1ull << 32) && h[2] < (1ull << 32),
               XAMG_ERR_INVALID_ARG, "hierarchy file: matrix sizes out of range");
    HCsr m;
    m.nrows = h[0];
    m.ncols = h[1];
    m.row.resize(h[0] + 1);
    m.col.resize(h[2]);
    m.val.resize(h[2]);
    read_exact(f, m.row.data(), m.row.size() * 4, "hierarchy row pointers");
    read_exact(f, m.col.data(), m.col.size() * 4, "hierarchy columns");
    read_exact(f, m.val.data(), m.val.size() * 8, "hierarchy values");
    XG_REQUIRE(m.row[0] == 0 && m.row[h[0]] == h[2], XAMG_ERR_INVALID_ARG,
               "hierarchy file: inconsistent row pointers");
    for (uint64_t i = 0; i < h[0]; ++i)
        XG_REQUIRE(m.row[i] <= m.row[i + 1], XAMG_ERR_INVALID_ARG,
                   "hierarchy file: row pointers decrease");
    for (uint32_t c : m.col)
        XG_REQUIRE(c < h[1], XAMG_ERR_INVALID_ARG, "hierarchy file: column out of range");
    return m;
}

}  // namespace

SystemSize read_system_size(const char *path) {
    XG_REQUIRE(path, XAMG_ERR_INVALID_ARG, "null path");
    File f(path, "rb");
    XG_REQUIRE(f.f, XAMG_ERR_INVALID_ARG, std::string("cannot open ") + path);
    uint32_t h[2];
    read_exact(f.f, h, sizeof(h), "the header");
    return SystemSize{h[0], h[1]};
}

int read_system(const char *path, int nv, uint32_t *row, uint32_t *col, double *val, double *b,
                double *x) {
    XG_REQUIRE(path && row && col && val, XAMG_ERR_INVALID_ARG, "null argument");
    File f(path, "rb");
    XG_REQUIRE(f.f, XAMG_ERR_INVALID_ARG, std::string("cannot open ") + path);
    const uint64_t size = file_size(f.f);
    uint32_t h[2];
    read_exact(f.f, h, sizeof(h), "the header");
    const uint64_t n = h[0], nnz = h[1];
    read_exact(f.f, row, (n + 1) * 4, "the row pointers");
    read_exact(f.f, col, nnz * 4, "the columns");
    read_exact(f.f, val, nnz * 8, "the values");
    XG_REQUIRE(row[0] == 0 && row[n] == nnz, XAMG_ERR_INVALID_ARG,
               "row pointers do not span the nonzeros");
    // b and x follow, [n][nv] interleaved; absent vectors take b = 1, x = 0
    // (reader.inl:155-172)
    const uint64_t pos = 8 + (n + 1) * 4 + nnz * 12, vb = n * (uint64_t)nv * 8;
    int found = 0;
    if (b) {
        if (size >= pos + vb) {
            read_exact(f.f, b, vb, "b");
            found |= 1;
        } else {
            for (uint64_t i = 0; i < n * (uint64_t)nv; ++i) b[i] = 1.0;
        }
    }
    if (x) {
        if ((found & 1) && size >= pos + 2 * vb) {
            read_exact(f.f, x, vb, "x");
            found |= 2;
        } else {
            std::memset(x, 0, vb);
        }
    }
    return found;
}

void write_system(const char *path, uint32_t nrows, uint32_t nnz, const uint32_t *row,
                  const uint32_t *col, const double *val, int nv, const double *b,
                  const double *x) {
    XG_REQUIRE(path && row && (nnz == 0 || (col && val)), XAMG_ERR_INVALID_ARG, "null argument");
    XG_REQUIRE(!x || b, XAMG_ERR_INVALID_ARG, "x is stored after b: give b too");
    XG_REQUIRE(row[0] == 0 && row[nrows] == nnz, XAMG_ERR_INVALID_ARG,
               "row pointers do not span the nonzeros");
    File f(path, "wb");
    XG_REQUIRE(f.f, XAMG_ERR_INVALID_ARG, std::string("cannot create ") + path);
    const uint32_t h[2] = {nrows, nnz};
    write_exact(f.f, h, sizeof(h));
    write_exact(f.f, row, ((uint64_t)nrows + 1) * 4);
    write_exact(f.f, col, (uint64_t)nnz * 4);
    write_exact(f.f, val, (uint64_t)nnz * 8);
    if (b) write_exact(f.f, b, (uint64_t)nrows * nv * 8);
    if (x) write_exact(f.f, x, (uint64_t)nrows * nv * 8);
}

uint64_t matrix_fingerprint(const HCsr &m) {
    uint64_t h = 1469598103934665603ull;
    const uint64_t s[3] = {m.nrows, m.ncols, (uint64_t)m.col.size()};
    h = fnv1a(h, s, sizeof(s));
    h = fnv1a(h, m.row.data(), m.row.size() * 4);
    h = fnv1a(h, m.col.data(), m.col.size() * 4);
    h = fnv1a(h, m.val.data(), m.val.size() * 8);
    return h;
}

void save_hierarchy(const char *path, const std::string &key, const HCsr &A0,
                    const Hierarchy &H) {
    XG_REQUIRE(path, XAMG_ERR_INVALID_ARG, "null path");
    File f(path, "wb");
    XG_REQUIRE(f.f, XAMG_ERR_INVALID_ARG, std::string("cannot create ") + path);
    write_exact(f.f, MAGIC, sizeof(MAGIC));
    const uint32_t hdr[2] = {VERSION, (uint32_t)key.size()};
    write_exact(f.f, hdr, sizeof(hdr));
    write_exact(f.f, key.data(), key.size());
    const uint64_t fp[3] = {A0.nrows, (uint64_t)A0.col.size(), matrix_fingerprint(A0)};
    write_exact(f.f, fp, sizeof(fp));
    const uint32_t nl = (uint32_t)H.lv.size();
    write_exact(f.f, &nl, 4);
    for (size_t li = 0; li < H.lv.size(); ++li) {
        const HLevel &l = H.lv[li];
        const double e[2] = {l.min_eig, l.max_eig};
        write_exact(f.f, e, sizeof(e));
        if (li > 0) write_csr(f.f, l.A);  // level 0 is the matrix itself
        const uint32_t hasP = l.P.nrows ? 1u : 0u;
        write_exact(f.f, &hasP, 4);
        if (hasP) write_csr(f.f, l.P);
    }
}

std::shared_ptr<const Hierarchy> load_hierarchy(const char *path, const HCsr &A0,
                                                std::string &key) {
    XG_REQUIRE(path, XAMG_ERR_INVALID_ARG, "null path");
    File f(path, "rb");
    XG_REQUIRE(f.f, XAMG_ERR_INVALID_ARG, std::string("cannot open ") + path);
    char magic[8];
    read_exact(f.f, magic, 8, "the header");
    XG_REQUIRE(std::memcmp(magic, MAGIC, 8) == 0, XAMG_ERR_INVALID_ARG,
               "not a hierarchy file of this library");
    uint32_t hdr[2];
    read_exact(f.f, hdr, sizeof(hdr), "the header");
    XG_REQUIRE(hdr[0] == VERSION, XAMG_ERR_UNSUPPORTED, "hierarchy file version not supported");
    XG_REQUIRE(hdr[1] < 4096, XAMG_ERR_INVALID_ARG, "hierarchy file: bad key length");
    key.assign(hdr[1], '\0');
    read_exact(f.f, &key[0], hdr[1], "the parameter key");
    uint64_t fp[3];
    read_exact(f.f, fp, sizeof(fp), "the matrix fingerprint");
    XG_REQUIRE(fp[0] == A0.nrows && fp[1] == A0.col.size() && fp[2] == matrix_fingerprint(A0),
               XAMG_ERR_INVALID_ARG, "the hierarchy file was built for another matrix");
    uint32_t nl = 0;
    read_exact(f.f, &nl, 4, "the level count");
    XG_REQUIRE(nl >= 1 && nl <= 64, XAMG_ERR_INVALID_ARG, "hierarchy file: bad level count");
    auto H = std::make_shared<Hierarchy>();
    H->lv.resize(nl);
    for (uint32_t l = 0; l < nl; ++l) {
        double e[2];
        read_exact(f.f, e, sizeof(e), "eigenvalue estimates");
        H->lv[l].min_eig = e[0];
        H->lv[l].max_eig = e[1];
        if (l > 0)
            H->lv[l].A = read_csr(f.f);
        else
            H->lv[0].A = A0;
        uint32_t hasP = 0;
        read_exact(f.f, &hasP, 4, "a level record");
        if (hasP) H->lv[l].P = read_csr(f.f);
    }
    // the levels must chain: A_l square, P_l maps level l+1 onto level l
    for (uint32_t l = 0; l < nl; ++l) {
        const HLevel &v = H->lv[l];
        XG_REQUIRE(v.A.nrows == v.A.ncols, XAMG_ERR_INVALID_ARG, "hierarchy file: A not square");
        if (l + 1 < nl)
            XG_REQUIRE(v.P.nrows == v.A.nrows && v.P.ncols == H->lv[l + 1].A.nrows,
                       XAMG_ERR_INVALID_ARG, "hierarchy file: P does not chain the levels");
    }
    XG_REQUIRE(H->lv[0].A.nrows == A0.nrows, XAMG_ERR_INVALID_ARG,
               "hierarchy file: level 0 differs from the matrix");
    return H;
}

}  // namespace xg
