// The reference's binary model file (.prn): loader() / saver() with
// fl1itp / fl1otp = 1 (pardiso/load3mg.c:745-905 read, 1298-1443 write).
// Host code only; the C ABI is in include/p2cuda.h.
//
// Layout, in the byte order and type sizes of the writing machine (the
// first four bytes record sizeof int, long, float, double; a reader with
// other sizes refuses the file, as the reference does):
//   header   xnumx ynumy znumz mnumx mnumy mnumz (long), xsize ysize zsize
//            (double), pxinit pyinit pzinit (long), pinit GXKOEF GYKOEF
//            GZKOEF (double), rocknum (int), bondnum marknum (long), cycle
//            (int), timesum in years, gridcur, gridtot (double)
//   rocks    24 tables of rocknum doubles: markn0 markn1 marks0 marks1 marknu
//            markdh markdv markss markmm markll marka0 marka1 markb0 markb1
//            marke0 marke1 markro markbb markaa markcp markkt markkf markkp
//            markht
//   nodes    per node 11 floats: pr vx vy vz ro nu tk cp et kt ht
//   grid     gx (xnumx floats), gy, gz
//   bonds    per boundary row: bondm index (long), row (long), const koef
//            (2 floats), bondn1 of the row (long)
//   markers  per marker 7 floats x y z markk markw markd marke, then the type
//            (one byte)
#include <cerrno>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <memory>

#include "../../include/p2cuda.h"

namespace {

p2_status fail(char *err, long errlen, p2_status code, const char *fmt, ...)
{
    if (err && errlen > 0) {
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(err, (size_t)errlen, fmt, ap);
        va_end(ap);
    }
    return code;
}

struct File {
    FILE *f = nullptr;
    ~File() { if (f) fclose(f); }
};

// every count read or written must come out whole
struct Io {
    FILE *f;
    bool ok = true;
    template <typename T>
    void rd(T *p, size_t n) { if (ok && n && fread(p, sizeof(T), n, f) != n) ok = false; }
    template <typename T>
    void wr(const T *p, size_t n) { if (ok && n && fwrite(p, sizeof(T), n, f) != n) ok = false; }
};

void header_io(Io &io, p2_prn_header *h, bool write)
{
    long *l6[6] = {&h->xnumx, &h->ynumy, &h->znumz, &h->mnumx, &h->mnumy, &h->mnumz};
    double *d3[3] = {&h->xsize, &h->ysize, &h->zsize};
    long *p3[3] = {&h->pxinit, &h->pyinit, &h->pzinit};
    double *d4[4] = {&h->pinit, &h->gxkoef, &h->gykoef, &h->gzkoef};
    for (long *p : l6) write ? io.wr(p, 1) : io.rd(p, 1);
    for (double *p : d3) write ? io.wr(p, 1) : io.rd(p, 1);
    for (long *p : p3) write ? io.wr(p, 1) : io.rd(p, 1);
    for (double *p : d4) write ? io.wr(p, 1) : io.rd(p, 1);
    write ? io.wr(&h->rocknum, 1) : io.rd(&h->rocknum, 1);
    write ? io.wr(&h->bondnum, 1) : io.rd(&h->bondnum, 1);
    write ? io.wr(&h->marknum, 1) : io.rd(&h->marknum, 1);
    write ? io.wr(&h->cycle, 1) : io.rd(&h->cycle, 1);
    write ? io.wr(&h->timesum_years, 1) : io.rd(&h->timesum_years, 1);
    write ? io.wr(&h->gridcur, 1) : io.rd(&h->gridcur, 1);
    write ? io.wr(&h->gridtot, 1) : io.rd(&h->gridtot, 1);
}

p2_status check_header(const p2_prn_header *h, char *err, long errlen)
{
    if (h->xnumx < 2 || h->ynumy < 2 || h->znumz < 2 || h->xnumx > (1L << 20) || h->ynumy > (1L << 20) ||
        h->znumz > (1L << 20))
        return fail(err, errlen, P2_ERR_ARG, "grid %ld x %ld x %ld out of range", h->xnumx, h->ynumy, h->znumz);
    if (h->rocknum < 0 || h->rocknum > 100000 || h->bondnum < 0 || h->marknum < 0)
        return fail(err, errlen, P2_ERR_ARG, "negative or too large counts (rocknum %d, bondnum %ld, marknum %ld)",
                    h->rocknum, h->bondnum, h->marknum);
    return P2_OK;
}

p2_status open_checked(File &F, const char *path, const char *mode, char *err, long errlen)
{
    if (!path) return fail(err, errlen, P2_ERR_ARG, "null path");
    F.f = fopen(path, mode);
    if (!F.f) return fail(err, errlen, P2_ERR_ARG, "cannot open %s: %s", path, strerror(errno));
    return P2_OK;
}

p2_status read_sizes(Io &io, char *err, long errlen)
{
    const char want[4] = {(char)sizeof(int), (char)sizeof(long), (char)sizeof(float), (char)sizeof(double)};
    const char *names[4] = {"INT", "LONG INT", "FLOAT", "DOUBLE"};
    char got[4];
    io.rd(got, 4);
    if (!io.ok) return fail(err, errlen, P2_ERR_ARG, "file shorter than its size bytes");
    for (int q = 0; q < 4; q++)
        if (got[q] != want[q])
            return fail(err, errlen, P2_ERR_ARG, "current %s size <%d> is different from given in file <%d>",
                        names[q], want[q], got[q]);
    return P2_OK;
}

}  // namespace

extern "C" p2_status p2_prn_read_header(const char *path, p2_prn_header *h, char *err, long errlen)
{
    if (err && errlen > 0) err[0] = 0;
    if (!h) return fail(err, errlen, P2_ERR_ARG, "null header");
    File F;
    p2_status st = open_checked(F, path, "rb", err, errlen);
    if (st) return st;
    Io io{F.f};
    if ((st = read_sizes(io, err, errlen))) return st;
    header_io(io, h, false);
    if (!io.ok) return fail(err, errlen, P2_ERR_ARG, "%s: truncated header", path);
    return check_header(h, err, errlen);
}

extern "C" p2_status p2_prn_read(const char *path, const p2_prn_header *h, const p2_prn_data *d, char *err,
                                 long errlen)
{
    if (err && errlen > 0) err[0] = 0;
    if (!h || !d) return fail(err, errlen, P2_ERR_ARG, "null header or data");
    p2_status st = check_header(h, err, errlen);
    if (st) return st;
    const long nodes = h->xnumx * h->ynumy * h->znumz;
    if (!d->rocks || !d->nodes || !d->gx || !d->gy || !d->gz ||
        (h->bondnum && (!d->bond_index || !d->bond_row || !d->bond_value || !d->bond_target)) ||
        (h->marknum && (!d->markers || !d->markt)))
        return fail(err, errlen, P2_ERR_ARG, "null array for a non-empty section");
    File F;
    if ((st = open_checked(F, path, "rb", err, errlen))) return st;
    Io io{F.f};
    if ((st = read_sizes(io, err, errlen))) return st;
    p2_prn_header hf;
    header_io(io, &hf, false);
    if (!io.ok) return fail(err, errlen, P2_ERR_ARG, "%s: truncated header", path);
    if (hf.xnumx != h->xnumx || hf.ynumy != h->ynumy || hf.znumz != h->znumz || hf.rocknum != h->rocknum ||
        hf.bondnum != h->bondnum || hf.marknum != h->marknum)
        return fail(err, errlen, P2_ERR_ARG, "%s: sizes differ from the header passed in", path);
    io.rd(d->rocks, (size_t)24 * h->rocknum);
    io.rd(d->nodes, (size_t)11 * nodes);
    io.rd(d->gx, (size_t)h->xnumx);
    io.rd(d->gy, (size_t)h->ynumy);
    io.rd(d->gz, (size_t)h->znumz);
    for (long q = 0; q < h->bondnum && io.ok; q++) {
        io.rd(d->bond_index + q, 1);
        io.rd(d->bond_row + q, 1);
        io.rd(d->bond_value + 2 * q, 2);
        io.rd(d->bond_target + q, 1);
    }
    for (long q = 0; q < h->marknum && io.ok; q++) {
        io.rd(d->markers + 7 * q, 7);
        io.rd(d->markt + q, 1);
    }
    if (!io.ok) return fail(err, errlen, P2_ERR_ARG, "%s: file ends before its sections do", path);
    return P2_OK;
}

extern "C" p2_status p2_prn_write(const char *path, const p2_prn_header *h, const p2_prn_data *d, char *err,
                                  long errlen)
{
    if (err && errlen > 0) err[0] = 0;
    if (!h || !d) return fail(err, errlen, P2_ERR_ARG, "null header or data");
    p2_status st = check_header(h, err, errlen);
    if (st) return st;
    const long nodes = h->xnumx * h->ynumy * h->znumz;
    if (!d->rocks || !d->nodes || !d->gx || !d->gy || !d->gz ||
        (h->bondnum && (!d->bond_index || !d->bond_row || !d->bond_value || !d->bond_target)) ||
        (h->marknum && (!d->markers || !d->markt)))
        return fail(err, errlen, P2_ERR_ARG, "null array for a non-empty section");
    File F;
    if ((st = open_checked(F, path, "wb", err, errlen))) return st;
    Io io{F.f};
    const char sizes[4] = {(char)sizeof(int), (char)sizeof(long), (char)sizeof(float), (char)sizeof(double)};
    io.wr(sizes, 4);
    p2_prn_header hc = *h;
    header_io(io, &hc, true);
    io.wr(d->rocks, (size_t)24 * h->rocknum);
    io.wr(d->nodes, (size_t)11 * nodes);
    io.wr(d->gx, (size_t)h->xnumx);
    io.wr(d->gy, (size_t)h->ynumy);
    io.wr(d->gz, (size_t)h->znumz);
    for (long q = 0; q < h->bondnum && io.ok; q++) {
        io.wr(d->bond_index + q, 1);
        io.wr(d->bond_row + q, 1);
        io.wr(d->bond_value + 2 * q, 2);
        io.wr(d->bond_target + q, 1);
    }
    for (long q = 0; q < h->marknum && io.ok; q++) {
        io.wr(d->markers + 7 * q, 7);
        io.wr(d->markt + q, 1);
    }
    if (!io.ok) return fail(err, errlen, P2_ERR_ARG, "%s: write failed: %s", path, strerror(errno));
    if (fclose(F.f) != 0) {
        F.f = nullptr;
        return fail(err, errlen, P2_ERR_ARG, "%s: close failed: %s", path, strerror(errno));
    }
    F.f = nullptr;
    return P2_OK;
}
