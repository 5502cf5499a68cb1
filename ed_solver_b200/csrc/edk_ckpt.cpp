// Eigenstate checkpoints (GS.raw) and the sector-bound file of the
// reference's solver, both list-directed Fortran text:
//   write_raw_eigensectorlist / read_raw_eigensectorlist (eigen_sector_class.f90:514-567)
//   write_raw_sector / read_raw_sector (quantum_sector_class.f90:174-212)
//   write_raw_fermion_sector(2) (quantum_fermion_sector_class.f90:398-425,
//   quantum_fermion_hilbert_class.f90:190-215)
//   write_raw_eigenlist / read_raw_eigenlist (eigen_class.f90:479-514)
//   write_raw_rcvector / read_raw_rcvector (rcvector_class.f90:217-248)
//   ed.sector_bound_file (solver.h:107-119 read, 396-402 write)
// Every WRITE(UNIT,*) of the reference is one record (line) here; the reader
// follows list-directed READ: a READ starts on a new record, takes its values
// across as many records as it needs, and drops the rest of its last record.
#include <cctype>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/edk.h"

namespace {

class ListReader {
public:
    explicit ListReader(FILE *f) : f_(f) {}

    // Start a READ statement: skip what is left of the current record.
    bool begin()
    {
        repeat_left_ = 0;
        if (!at_record_start_) {
            int c;
            while ((c = getc(f_)) != EOF && c != '\n') {}
            if (c == EOF) return false;
        }
        at_record_start_ = false;
        return true;
    }

    // Next value of the current READ.
    bool token(std::string &t)
    {
        if (repeat_left_ > 0) { --repeat_left_; t = repeat_tok_; return true; }
        int c;
        for (;;) {
            c = getc(f_);
            if (c == EOF) return false;
            if (c == ' ' || c == '\t' || c == '\r' || c == ',' || c == '\n') continue;
            break;
        }
        at_record_start_ = false;      // inside the record this value starts in
        t.clear();
        if (c == '\'' || c == '"') {
            const int q = c;
            for (;;) {
                c = getc(f_);
                if (c == EOF) return false;
                if (c == q) {
                    const int d = getc(f_);
                    if (d == q) { t.push_back((char)q); continue; }   // doubled quote
                    if (d != EOF) ungetc(d, f_);
                    break;
                }
                if (c == '\n') continue;
                t.push_back((char)c);
            }
            end_token();
            return true;
        }
        while (c != EOF && c != ' ' && c != '\t' && c != '\r' && c != ',' && c != '\n') {
            t.push_back((char)c);
            c = getc(f_);
        }
        if (c == '\n') at_record_start_ = true;
        // r*c: the value c repeated r times
        const size_t star = t.find('*');
        if (star != std::string::npos && star > 0) {
            bool digits = true;
            for (size_t i = 0; i < star; ++i) digits = digits && std::isdigit((unsigned char)t[i]);
            if (digits) {
                const long long r = std::atoll(t.substr(0, star).c_str());
                std::string v = t.substr(star + 1);
                if (r < 1 || v.empty()) return false;          // null values are not used by these files
                repeat_tok_ = v;
                repeat_left_ = r - 1;
                t = v;
            }
        }
        return true;
    }

    bool logical(bool &v)
    {
        std::string t;
        if (!token(t)) return false;
        size_t i = t[0] == '.' ? 1 : 0;
        if (i >= t.size()) return false;
        const char c = (char)std::toupper((unsigned char)t[i]);
        if (c == 'T') { v = true; return true; }
        if (c == 'F') { v = false; return true; }
        return false;
    }
    bool integer(long long &v)
    {
        std::string t;
        if (!token(t)) return false;
        char *end = nullptr;
        v = std::strtoll(t.c_str(), &end, 10);
        return end && *end == '\0';
    }
    bool real(double &v)
    {
        std::string t;
        if (!token(t)) return false;
        for (auto &ch : t)
            if (ch == 'd' || ch == 'D') ch = 'E';
        char *end = nullptr;
        v = std::strtod(t.c_str(), &end);
        return end && *end == '\0';
    }
    bool word(std::string &v) { return token(v); }

    // The read completed at a record end already consumed (the next READ
    // must not skip another record).
    void end_token()
    {
        const int c = getc(f_);
        if (c == '\n') at_record_start_ = true;
        else if (c != EOF) ungetc(c, f_);
    }

private:
    FILE *f_;
    bool at_record_start_ = true;
    long long repeat_left_ = 0;
    std::string repeat_tok_;
};

struct File {
    FILE *f = nullptr;
    ~File() { if (f) std::fclose(f); }
};

bool same_sector(const edk_gs_entry &a, const edk_gs_entry &b)
{
    return a.kind == b.kind && a.norbs == b.norbs && a.nup == b.nup && a.ndn == b.ndn;
}

}  // namespace

extern "C" int edk_gs_write(const char *path, int32_t nentries, const edk_gs_entry *e, const double *pool)
{
    if (!path || nentries < 0 || (nentries > 0 && (!e || !pool))) return EDK_ERR_INVALID;
    for (int i = 0; i < nentries; ++i)
        if (e[i].n < 0 || e[i].offset < 0 || (e[i].kind != 0 && e[i].kind != 1)) return EDK_ERR_INVALID;
    std::vector<char> buf(1 << 20);   // declared first: it outlives the stream using it
    File out;
    out.f = std::fopen(path, "w");
    if (!out.f) return EDK_ERR_INVALID;
    std::setvbuf(out.f, buf.data(), _IOFBF, buf.size());
    FILE *f = out.f;
    auto logical = [&](bool v) { std::fprintf(f, " %c\n", v ? 'T' : 'F'); };
    auto integer = [&](long long v) { std::fprintf(f, " %11lld\n", v); };
    auto real = [&](double v) { std::fprintf(f, " %25.17E\n", v); };
    int i = 0;
    while (i < nentries) {
        logical(true);                                     // a new eigensector
        if (e[i].kind == 0) {
            std::fprintf(f, " updo\n");
            integer(e[i].norbs); integer(e[i].nup);
            integer(e[i].norbs); integer(e[i].ndn);
        } else {
            std::fprintf(f, " sz\n");
            integer(e[i].norbs); integer(e[i].nup);
        }
        int j = i;
        for (; j < nentries && same_sector(e[j], e[i]); ++j) {
            logical(true);                                 // a new eigenstate
            real(e[j].val);
            logical(e[j].converged != 0);
            integer(e[j].rank);
            integer(e[j].n);
            const double *v = pool + e[j].offset;
            for (int64_t q = 0; q < e[j].n; ++q)
                std::fprintf(f, (q % 4 == 3 || q + 1 == e[j].n) ? " %25.17E\n" : " %25.17E", v[q]);
            if (e[j].n == 0) std::fprintf(f, "\n");
        }
        logical(false);                                    // end of the eigenlist
        i = j;
    }
    logical(false);                                        // end of the list
    if (std::fflush(f) != 0) return EDK_ERR_INVALID;
    return EDK_OK;
}

extern "C" int edk_gs_read(const char *path, int32_t cap, edk_gs_entry *entries, int32_t *nentries, int64_t vec_cap,
                           double *pool, int64_t *vec_total)
{
    if (!path || !nentries || !vec_total) return EDK_ERR_INVALID;
    std::vector<char> buf(1 << 20);   // declared first: it outlives the stream using it
    File in;
    in.f = std::fopen(path, "r");
    if (!in.f) return EDK_ERR_INVALID;
    std::setvbuf(in.f, buf.data(), _IOFBF, buf.size());
    ListReader R(in.f);
    int32_t n = 0;
    int64_t used = 0;
    for (;;) {
        bool item = false;
        if (!R.begin() || !R.logical(item)) return EDK_ERR_INVALID;
        if (!item) break;
        edk_gs_entry sec{};
        std::string kind;
        if (!R.begin() || !R.word(kind)) return EDK_ERR_INVALID;
        long long norbs = 0, np = 0;
        auto fermion_sector = [&](long long &no, long long &npart) {
            return R.begin() && R.integer(no) && R.begin() && R.integer(npart);
        };
        if (kind.find("updo") != std::string::npos) {
            long long no2 = 0, np2 = 0;
            if (!fermion_sector(norbs, np) || !fermion_sector(no2, np2) || no2 != norbs) return EDK_ERR_INVALID;
            sec.kind = 0;
            sec.norbs = (int32_t)norbs;
            sec.nup = (int32_t)np;
            sec.ndn = (int32_t)np2;
        } else if (kind.find("sz") != std::string::npos) {
            if (!fermion_sector(norbs, np)) return EDK_ERR_INVALID;
            sec.kind = 1;
            sec.norbs = (int32_t)norbs;
            sec.nup = (int32_t)np;
            sec.ndn = -1;
        } else {
            return EDK_ERR_INVALID;
        }
        for (;;) {
            bool state = false;
            if (!R.begin() || !R.logical(state)) return EDK_ERR_INVALID;
            if (!state) break;
            edk_gs_entry en = sec;
            double val = 0.0;
            bool conv = false;
            long long rank = 0, len = 0;
            if (!R.begin() || !R.real(val)) return EDK_ERR_INVALID;
            if (!R.begin() || !R.logical(conv)) return EDK_ERR_INVALID;
            if (!R.begin() || !R.integer(rank)) return EDK_ERR_INVALID;
            if (!R.begin() || !R.integer(len) || len < 0) return EDK_ERR_INVALID;
            en.val = val;
            en.converged = conv ? 1 : 0;
            en.rank = (int32_t)rank;
            en.n = len;
            en.offset = used;
            if (!R.begin() && len > 0) return EDK_ERR_INVALID;
            const bool store = pool && used + len <= vec_cap;
            for (long long q = 0; q < len; ++q) {
                double x = 0.0;
                if (!R.real(x)) return EDK_ERR_INVALID;
                if (store) pool[used + q] = x;
            }
            if (entries && n < cap) entries[n] = en;
            ++n;
            used += len;
        }
    }
    *nentries = n;
    *vec_total = used;
    if (entries && n > cap) return EDK_ERR_INVALID;
    if (pool && used > vec_cap) return EDK_ERR_INVALID;
    return EDK_OK;
}

extern "C" int edk_sector_bounds_read(const char *path, int32_t *b, int32_t *has_sz)
{
    if (!path || !b) return EDK_ERR_INVALID;
    File in;
    in.f = std::fopen(path, "r");
    if (!in.f) return EDK_ERR_INVALID;
    ListReader R(in.f);
    long long v[6] = {0, 0, 0, 0, 1000, -1000};
    for (int r = 0; r < 2; ++r)
        if (!R.begin() || !R.integer(v[2 * r]) || !R.integer(v[2 * r + 1])) return EDK_ERR_INVALID;
    int sz = 0;
    long long a = 0, c = 0;
    if (R.begin() && R.integer(a) && R.integer(c)) { v[4] = a; v[5] = c; sz = 1; }   // READ(...,end=31)
    for (int i = 0; i < 6; ++i) b[i] = (int32_t)v[i];
    if (has_sz) *has_sz = sz;
    return EDK_OK;
}

extern "C" int edk_sector_bounds_write(const char *path, const int32_t *b)
{
    if (!path || !b) return EDK_ERR_INVALID;
    File out;
    out.f = std::fopen(path, "w");
    if (!out.f) return EDK_ERR_INVALID;
    for (int r = 0; r < 3; ++r) std::fprintf(out.f, " %11d %11d\n", b[2 * r], b[2 * r + 1]);
    return std::fflush(out.f) == 0 ? EDK_OK : EDK_ERR_INVALID;
}
