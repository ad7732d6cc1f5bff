// host_output.cpp -- clawpack 4.6 ASCII frames (fort.tXXXX header, fort.qXXXX patches)
// and VTK unstructured-grid files (<prefix>_frame_NNNN.vtu).
//
// fclaw2d_clawpatch_output_ascii.c:112-170 and fort_4.6/fclaw2d_clawpatch46_output_ascii.f:
//   fort.t: time (E30.20), meqn, ngrids, num_aux, num_dim (I5 + label)
//   fort.q: per patch, in the reference's patch order (block, then the leaves of
//           the block along the space-filling curve): grid_number, AMR_level,
//           block_number, mpi_rank, mx, my (I5 + label), xlow, ylow, dx, dy (E24.16
//           + label), a blank line, then for j = 1..my the rows i = 1..mx with the
//           meqn values of a cell on one line (E26.16 each, |q| < 1e-99 written as 0)
//           and a blank line after each row.
// The Fortran E format is restated here: 0.ddd...dE+xx (d digits after the point,
// correctly rounded), E dropped for three-digit exponents, right-justified.
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include "fc2d_b200.h"

namespace {

// Fortran Ew.d of v
std::string fortran_e(double v, int w, int d)
{
    char buf[64];
    std::string body;
    if (v == 0.0 || !std::isfinite(v)) {
        if (!std::isfinite(v)) body = std::isnan(v) ? "NaN" : (v > 0 ? "Infinity" : "-Infinity");
        else body = std::string(std::signbit(v) ? "-" : "") + "0." + std::string(d, '0') + "E+00";
    } else {
        // d significant digits: printf gives m.mmm (d-1 after the point) E e; Fortran
        // writes 0.mmmm E (e+1)
        std::snprintf(buf, sizeof(buf), "%.*E", d - 1, v);
        std::string s(buf);
        const size_t epos = s.find('E');
        std::string mant = s.substr(0, epos);
        const int e = std::atoi(s.c_str() + epos + 1) + 1;
        const bool neg = mant[0] == '-';
        if (neg) mant = mant.substr(1);
        std::string digits;
        for (char c : mant)
            if (c != '.') digits += c;
        char ex[16];
        if (std::abs(e) < 100) std::snprintf(ex, sizeof(ex), "E%c%02d", e < 0 ? '-' : '+', std::abs(e));
        else std::snprintf(ex, sizeof(ex), "%c%03d", e < 0 ? '-' : '+', std::abs(e));
        body = std::string(neg ? "-" : "") + "0." + digits + ex;
    }
    if ((int)body.size() >= w) return body;
    return std::string(w - body.size(), ' ') + body;
}

std::string fortran_i(int v, int w)
{
    char buf[32];
    std::snprintf(buf, sizeof(buf), "%*d", w, v);
    return buf;
}

}  // namespace

extern "C" int fc2d_b200_write_ascii_frame(const char* dir, int iframe, double time, int meqn, int maux, int mx, int my,
                                           int mbc, int npatch, const int* level, const int* block,
                                           const double* xlower, const double* ylower, const double* dx,
                                           const double* dy, const double* q)
{
    if (!dir || iframe < 0 || meqn <= 0 || meqn > 20 || mx <= 0 || my <= 0 || mbc < 0 || npatch < 0)
        return FC2D_B200_EINVAL;
    char name[32];
    std::snprintf(name, sizeof(name), "/fort.t%04d", iframe);
    FILE* ft = std::fopen((std::string(dir) + name).c_str(), "w");
    if (!ft) return FC2D_B200_EINVAL;
    std::fprintf(ft, "%s    time\n", fortran_e(time, 30, 20).c_str());
    std::fprintf(ft, "%s                 meqn\n", fortran_i(meqn, 5).c_str());
    std::fprintf(ft, "%s                 ngrids\n", fortran_i(npatch, 5).c_str());
    std::fprintf(ft, "%s                 num_aux\n", fortran_i(maux, 5).c_str());
    std::fprintf(ft, "%s                 num_dim\n", fortran_i(2, 5).c_str());
    std::fclose(ft);
    std::snprintf(name, sizeof(name), "/fort.q%04d", iframe);
    FILE* fq = std::fopen((std::string(dir) + name).c_str(), "w");
    if (!fq) return FC2D_B200_EINVAL;
    const int nx = mx + 2 * mbc, ny = my + 2 * mbc;
    const size_t nq = (size_t)nx * ny * meqn;
    for (int p = 0; p < npatch; p++) {
        std::fprintf(fq, "%s                 grid_number\n", fortran_i(p, 5).c_str());
        std::fprintf(fq, "%s                 AMR_level\n", fortran_i(level[p], 5).c_str());
        std::fprintf(fq, "%s                 block_number\n", fortran_i(block[p], 5).c_str());
        std::fprintf(fq, "%s                 mpi_rank\n", fortran_i(0, 5).c_str());
        std::fprintf(fq, "%s                 mx\n", fortran_i(mx, 5).c_str());
        std::fprintf(fq, "%s                 my\n", fortran_i(my, 5).c_str());
        std::fprintf(fq, "%s    xlow\n", fortran_e(xlower[p], 24, 16).c_str());
        std::fprintf(fq, "%s    ylow\n", fortran_e(ylower[p], 24, 16).c_str());
        std::fprintf(fq, "%s    dx\n", fortran_e(dx[p], 24, 16).c_str());
        std::fprintf(fq, "%s    dy\n\n", fortran_e(dy[p], 24, 16).c_str());
        const double* qp = q + (size_t)p * nq;
        for (int j = 1; j <= my; j++) {
            for (int i = 1; i <= mx; i++) {
                std::string line;
                for (int m = 0; m < meqn; m++) {
                    double v = qp[(size_t)m * nx * ny + (size_t)(j + mbc - 1) * nx + (i + mbc - 1)];
                    if (std::fabs(v) < 1e-99) v = 0.0;
                    line += fortran_e(v, 26, 16);
                }
                std::fprintf(fq, "%s\n", line.c_str());
            }
            std::fprintf(fq, "  \n");
        }
    }
    std::fclose(fq);
    return 0;
}

// ---------------------------------------------------------------------------
// VTK (fclaw2d_clawpatch_output_vtk.c): one <prefix>_frame_NNNN.vtu, an XML
// UnstructuredGrid with raw appended data -- per patch (mx+1)(my+1) points
// (Float64 x3), mx*my quads (VTK type 9) with their connectivity and offsets,
// the cell fields mpirank (Int32), blockno (Int32), patchno and the meqn fields
// as Float32 per cell.  Each appended array is preceded by its byte count
// (UInt64); integer arrays are Int32 when every index fits, else Int64
// (fclaw2d_vtk_write_file, :593-698; header :97-197; footer :564-591).
// ---------------------------------------------------------------------------
extern "C" int fc2d_b200_write_vtk_file(const char* path, int mx, int my, int meqn, int npatch, const int* block,
                                        const double* points, const float* values)
{
    if (!path || mx <= 0 || my <= 0 || meqn <= 0 || npatch < 0 || (npatch > 0 && (!block || !points || !values)))
        return FC2D_B200_EINVAL;
    const int64_t ppp = (int64_t)(mx + 1) * (my + 1), cpp = (int64_t)mx * my, np = npatch;
    const int64_t npts = ppp * np, ncells = cpp * np, nconn = 4 * (ncells + 1);
    const bool fits32 = npts <= INT32_MAX && nconn <= INT32_MAX;
    const char* inttype = fits32 ? "Int32" : "Int64";
    const int64_t isz = fits32 ? 4 : 8, nd = 8;
    const int64_t ps_pos = ppp * 3 * 8, ps_conn = cpp * 4 * isz, ps_off = cpp * isz, ps_typ = cpp,
                  ps_rank = cpp * 4, ps_blk = cpp * 4, ps_pno = cpp * isz, ps_q = cpp * meqn * 4;
    const int64_t o_pos = 0, o_conn = nd + o_pos + ps_pos * np, o_off = nd + o_conn + ps_conn * np,
                  o_typ = nd + o_off + ps_off * np, o_rank = nd + o_typ + ps_typ * np,
                  o_blk = nd + o_rank + ps_rank * np, o_pno = nd + o_blk + ps_blk * np,
                  o_q = nd + o_pno + ps_pno * np;
    FILE* f = std::fopen(path, "wb");
    if (!f) return FC2D_B200_EINVAL;
    bool bad = false;
    auto pr = [&](const char* fmt, auto... a) { if (!bad && std::fprintf(f, fmt, a...) < 0) bad = true; };
    pr("<?xml version=\"1.0\"?>\n");
    pr("<VTKFile type=\"UnstructuredGrid\" version=\"0.1\" byte_order=\"LittleEndian\" header_type=\"UInt64\" >\n");
    pr(" <UnstructuredGrid>\n");
    pr("  <Piece NumberOfPoints=\"%lld\" NumberOfCells=\"%lld\">\n", (long long)npts, (long long)ncells);
    pr("   <Points>\n");
    pr("    <DataArray type=\"Float64\" Name=\"Position\" NumberOfComponents=\"3\" format=\"appended\" offset=\"%lld\">\n",
       (long long)o_pos);
    pr("    </DataArray>\n");
    pr("   </Points>\n");
    pr("   <Cells>\n");
    pr("    <DataArray type=\"%s\" Name=\"connectivity\" format=\"appended\" offset=\"%lld\">\n", inttype,
       (long long)o_conn);
    pr("    </DataArray>\n");
    pr("    <DataArray type=\"%s\" Name=\"offsets\" format=\"appended\" offset=\"%lld\">\n", inttype,
       (long long)o_off);
    pr("    </DataArray>\n");
    pr("    <DataArray type=\"UInt8\" Name=\"types\" format=\"appended\" offset=\"%lld\">\n", (long long)o_typ);
    pr("    </DataArray>\n");
    pr("   </Cells>\n");
    pr("   <CellData Scalars=\"mpirank,blockno,patchno\" Fields=\"meqn\">\n");
    pr("    <DataArray type=\"Int32\" Name=\"mpirank\" format=\"appended\" offset=\"%lld\">\n", (long long)o_rank);
    pr("    </DataArray>\n");
    pr("    <DataArray type=\"Int32\" Name=\"blockno\" format=\"appended\" offset=\"%lld\">\n", (long long)o_blk);
    pr("    </DataArray>\n");
    pr("    <DataArray type=\"%s\" Name=\"patchno\" format=\"appended\" offset=\"%lld\">\n", inttype, (long long)o_pno);
    pr("    </DataArray>\n");
    if (meqn == 1)
        pr("    <DataArray type=\"Float32\" Name=\"meqn\" format=\"appended\" offset=\"%lld\">\n", (long long)o_q);
    else
        pr("    <DataArray type=\"Float32\" Name=\"meqn\" NumberOfComponents=\"%d\" format=\"appended\" offset=\"%lld\">\n",
           meqn, (long long)o_q);
    pr("    </DataArray>\n");
    pr("   </CellData>\n");
    pr("   <PointData>\n");
    pr("   </PointData>\n");
    pr("  </Piece>\n");
    pr(" </UnstructuredGrid>\n");
    pr(" <AppendedData encoding=\"raw\">\n  _");
    auto put = [&](const void* p, size_t n) { if (!bad && n && std::fwrite(p, n, 1, f) != 1) bad = true; };
    auto count = [&](int64_t psize) { const uint64_t c = (uint64_t)(psize * np); put(&c, 8); };
    std::vector<char> buf;
    // positions
    count(ps_pos);
    put(points, (size_t)(ps_pos * np));
    // connectivity: the quad of cell (i, j) over the patch's own points
    count(ps_conn);
    buf.resize((size_t)ps_conn);
    for (int64_t p = 0; p < np; p++) {
        const int64_t pb = ppp * p;
        int64_t t = 0;
        for (int j = 0; j < my; j++)
            for (int i = 0; i < mx; i++) {
                const int64_t l = pb + i + (int64_t)j * (mx + 1);
                const int64_t v[4] = {l, l + 1, l + (mx + 2), l + (mx + 1)};
                for (int c = 0; c < 4; c++, t++) {
                    if (fits32) { const int32_t x = (int32_t)v[c]; std::memcpy(&buf[t * 4], &x, 4); }
                    else std::memcpy(&buf[t * 8], &v[c], 8);
                }
            }
        put(buf.data(), buf.size());
    }
    // offsets: 4 (cell index + 1)
    count(ps_off);
    buf.resize((size_t)ps_off);
    for (int64_t p = 0; p < np; p++) {
        for (int64_t c = 0; c < cpp; c++) {
            const int64_t k = 4 * (cpp * p + c + 1);
            if (fits32) { const int32_t x = (int32_t)k; std::memcpy(&buf[c * 4], &x, 4); }
            else std::memcpy(&buf[c * 8], &k, 8);
        }
        put(buf.data(), buf.size());
    }
    // types: VTK_QUAD
    count(ps_typ);
    buf.assign((size_t)ps_typ, (char)9);
    for (int64_t p = 0; p < np; p++) put(buf.data(), buf.size());
    // mpirank, blockno, patchno
    count(ps_rank);
    buf.assign((size_t)ps_rank, 0);
    for (int64_t p = 0; p < np; p++) put(buf.data(), buf.size());
    count(ps_blk);
    buf.resize((size_t)ps_blk);
    for (int64_t p = 0; p < np; p++) {
        const int32_t b = block[p];
        for (int64_t c = 0; c < cpp; c++) std::memcpy(&buf[c * 4], &b, 4);
        put(buf.data(), buf.size());
    }
    count(ps_pno);
    buf.resize((size_t)ps_pno);
    for (int64_t p = 0; p < np; p++) {
        for (int64_t c = 0; c < cpp; c++) {
            if (fits32) { const int32_t x = (int32_t)p; std::memcpy(&buf[c * 4], &x, 4); }
            else std::memcpy(&buf[c * 8], &p, 8);
        }
        put(buf.data(), buf.size());
    }
    // the fields, cell by cell, meqn values each
    count(ps_q);
    put(values, (size_t)(ps_q * np));
    pr("\n </AppendedData>\n</VTKFile>\n");
    if (std::fclose(f) != 0) bad = true;
    return bad ? FC2D_B200_EINVAL : 0;
}
