// Dataset import with the reference's parse rules and point order.
//
// importNDDataset (import_dataset.cpp:34-72) splits the file on ',' only and
// reads every whitespace-separated number inside each piece with
// `stringstream >> double`, stopping at the first piece that fails to parse;
// the flat list is cut into points of GPUNUMDIM values (a trailing partial
// point is dropped).  sortInNDBins (import_dataset.cpp:16-30, 76-80) then runs
// std::sort (not stable) with a comparator on int(coordinate) per dimension.
// Ids in the join are positions after that sort, so it is replayed here with
// the same comparator over an index array: std::sort's element moves depend
// only on comparison outcomes, so the permutation is the reference's.  The
// parse runs on all host threads (pieces are independent); the sort itself
// stays one std::sort, which is what fixes the permutation.
#include <algorithm>
#include <omp.h>
#include <cctype>
#include <cerrno>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

namespace sj {

// Accepts the grammar std::num_get accepts for double: [+-]digits[.digits][(e|E)[+-]digits]
// (also ".5" and "5."), converted with strtod (which libstdc++ uses underneath).
// Returns false when no number starts at p.
static bool parse_number(const char *&p, const char *end, double &out)
{
    const char *s = p;
    char buf[128];
    int n = 0;
    auto push = [&](char c) { if (n < 127) buf[n++] = c; };
    if (s < end && (*s == '+' || *s == '-')) push(*s++);
    int digits = 0;
    while (s < end && isdigit((unsigned char)*s)) { push(*s++); digits++; }
    if (s < end && *s == '.') {
        push(*s++);
        while (s < end && isdigit((unsigned char)*s)) { push(*s++); digits++; }
    }
    if (digits == 0) return false;
    if (s < end && (*s == 'e' || *s == 'E')) {
        const char *e = s + 1;
        char eb[64];
        int en = 0;
        eb[en++] = *s;
        if (e < end && (*e == '+' || *e == '-')) eb[en++] = *e++;
        int ed = 0;
        while (e < end && isdigit((unsigned char)*e) && en < 60) { eb[en++] = *e++; ed++; }
        if (ed == 0) return false;   // "1e" fails the stream extraction as a whole
        for (int i = 0; i < en; i++) push(eb[i]);
        s = e;
    }
    buf[n] = 0;
    errno = 0;
    out = strtod(buf, nullptr);
    p = s;
    return true;
}

// Parses the comma-separated pieces of [p, end) (end is the file end or just
// after a comma) in order, appending every number to out.
static void parse_pieces(const char *p, const char *end, std::vector<double> &out)
{
    while (p < end) {
        const char *tokEnd = (const char *)memchr(p, ',', (size_t)(end - p));
        if (!tokEnd) tokEnd = end;
        const char *q = p;
        for (;;) {
            while (q < tokEnd && isspace((unsigned char)*q)) q++;
            if (q >= tokEnd) break;
            double v;
            if (!parse_number(q, tokEnd, v)) break;
            out.push_back(v);
            // stream.peek() == ',' cannot happen inside a piece split on ','
        }
        p = (tokEnd < end) ? tokEnd + 1 : end;
    }
}

int import_csv(const char *path, int D, std::vector<double> &pts)
{
    FILE *f = fopen(path, "rb");
    if (!f) return -1;
    std::vector<char> data;
    {
        fseek(f, 0, SEEK_END);
        long sz = ftell(f);
        fseek(f, 0, SEEK_SET);
        if (sz < 0) { fclose(f); return -1; }
        data.resize((size_t)sz);
        if (sz > 0 && fread(data.data(), 1, (size_t)sz, f) != (size_t)sz) { fclose(f); return -1; }
    }
    fclose(f);
    // Pieces (text between commas) parse independently, so the file is cut
    // just after commas into one range per thread and the ranges' numbers are
    // concatenated in file order: the same flat list as a sequential parse.
    const char *base = data.data(), *end = base + data.size();
    const int T = std::max(1, std::min(omp_get_max_threads(), (int)(data.size() / (1 << 20)) + 1));
    std::vector<const char *> cut(T + 1);
    cut[0] = base;
    cut[T] = end;
    for (int t = 1; t < T; t++) {
        const char *c = std::max(cut[t - 1], base + data.size() * (size_t)t / (size_t)T);
        const char *comma = (c < end) ? (const char *)memchr(c, ',', (size_t)(end - c)) : nullptr;
        cut[t] = comma ? comma + 1 : end;
    }
    std::vector<std::vector<double>> part(T);
#pragma omp parallel for schedule(static, 1) num_threads(T)
    for (int t = 0; t < T; t++) {
        part[t].reserve((size_t)(cut[t + 1] - cut[t]) / 8 + 16);
        parse_pieces(cut[t], cut[t + 1], part[t]);
    }
    std::vector<size_t> off(T + 1, 0);
    for (int t = 0; t < T; t++) off[t + 1] = off[t] + part[t].size();
    const size_t npts = off[T] / (size_t)D;   // a trailing partial point is dropped
    std::vector<double> flat(npts * (size_t)D);
#pragma omp parallel for schedule(static, 1) num_threads(T)
    for (int t = 0; t < T; t++) {
        const size_t b = std::min(off[t], flat.size()), e = std::min(off[t + 1], flat.size());
        if (e > b) memcpy(flat.data() + b, part[t].data(), sizeof(double) * (e - b));
    }
    part.clear();
    // sortInNDBins replay: the comparator reads each point's int() bins,
    // computed once (same comparison outcomes, so the same permutation)
    std::vector<int> bins(npts * (size_t)D);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)(npts * (size_t)D); i++) bins[i] = int(flat[i]);
    std::vector<uint32_t> idx(npts);
    for (size_t i = 0; i < npts; i++) idx[i] = (uint32_t)i;
    const int *bb = bins.data();
    std::sort(idx.begin(), idx.end(), [bb, D](uint32_t a, uint32_t b) {
        const int *pa = bb + (size_t)a * D, *pb = bb + (size_t)b * D;
        for (int i = 0; i < D; i++) {
            if (pa[i] < pb[i]) return true;
            if (pa[i] > pb[i]) return false;
        }
        return false;
    });
    pts.resize(npts * (size_t)D);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)npts; i++)
        memcpy(&pts[(size_t)i * D], &flat[(size_t)idx[i] * D], sizeof(double) * (size_t)D);
    return 0;
}

}  // namespace sj
