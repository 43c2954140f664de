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
// only on comparison outcomes, so the permutation is the reference's.
#include <algorithm>
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
    std::vector<double> flat;
    flat.reserve(data.size() / 8);
    const char *p = data.data(), *end = p + data.size();
    while (p < end) {
        const char *tokEnd = (const char *)memchr(p, ',', (size_t)(end - p));
        if (!tokEnd) tokEnd = end;
        const char *q = p;
        for (;;) {
            while (q < tokEnd && isspace((unsigned char)*q)) q++;
            if (q >= tokEnd) break;
            double v;
            if (!parse_number(q, tokEnd, v)) break;
            flat.push_back(v);
            // stream.peek() == ',' cannot happen inside a piece split on ','
        }
        p = (tokEnd < end) ? tokEnd + 1 : end;
    }
    size_t npts = flat.size() / (size_t)D;
    flat.resize(npts * (size_t)D);
    // sortInNDBins replay
    std::vector<uint32_t> idx(npts);
    for (size_t i = 0; i < npts; i++) idx[i] = (uint32_t)i;
    const double *x = flat.data();
    std::sort(idx.begin(), idx.end(), [x, D](uint32_t a, uint32_t b) {
        for (int i = 0; i < D; i++) {
            int ia = int(x[(size_t)a * D + i]), ib = int(x[(size_t)b * D + i]);
            if (ia < ib) return true;
            if (ia > ib) return false;
        }
        return false;
    });
    pts.resize(npts * (size_t)D);
    for (size_t i = 0; i < npts; i++)
        memcpy(&pts[i * D], &flat[(size_t)idx[i] * D], sizeof(double) * (size_t)D);
    return 0;
}

}  // namespace sj
