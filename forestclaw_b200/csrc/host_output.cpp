// host_output.cpp -- clawpack 4.6 ASCII frames (fort.tXXXX header, fort.qXXXX patches).
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
#include <cmath>
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
