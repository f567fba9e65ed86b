/*
 * ref_io.cpp -- runs the reference's OWN configuration-file readers and writers on the host, to
 * pin the file-format restatement of the oracle.  TEST INFRASTRUCTURE ONLY.  Compiled by
 * oracle/Makefile against the reference tree (read in place, never copied) into
 * oracle/_ref/libref_io.so, for one compile-time lattice (the reference's GlobalConstants.h
 * takes the extents from _T_, _X_, _Y_, _Z_).
 *
 * What comes from the reference, unmodified, through #include:
 *   lattice/LinkFile.hxx, lattice/filetypes/{FilePlain,FileVogt,FileHeaderOnly}.hxx,
 *   lattice/access_pattern/{StandardPattern,GpuPattern}.hxx, lattice/SiteCoord.hxx,
 *   gaugefixing/apps/ildg.cpp (readILDG / writeILDG), gaugefixing/apps/qcdstag.cpp
 *   (readQCDSTAG / writeQCDSTAG) and, compiled beside it as C, the c-lime sources those use.
 * What this file adds: extern "C" wrappers with the pattern types the reference drivers use
 * (apps/LandauGaugeFixingSU3_4D.cu:53-54,119-121; the Coulomb apps' GpuPatternTimeslice,
 * apps/CoulombGaugeFixingSU3_4D.cu:57-59), and oracle/shim/boost (boost::iequals).
 */
#define __constant__
#include <cstdint>
#include <cstdio>
#include <iostream>
#include <sstream>

#include "lattice/LinkFile.hxx"
#include "lattice/SiteCoord.hxx"
#include "lattice/access_pattern/GpuPattern.hxx"
#include "lattice/access_pattern/GpuPatternTimeslice.hxx"
#include "lattice/access_pattern/StandardPattern.hxx"
#include "lattice/filetypes/FileHeaderOnly.hxx"
#include "lattice/filetypes/FilePlain.hxx"
#include "lattice/filetypes/FileVogt.hxx"
#include "gaugefixing/apps/ildg.cpp"
#include "gaugefixing/apps/qcdstag.cpp"

typedef StandardPattern<SiteCoord<4, NO_SPLIT>, 4, 3> RefStandard;
typedef GpuPattern<SiteCoord<4, FULL_SPLIT>, 4, 3> RefGpu;
typedef GpuPatternTimeslice<SiteCoord<4, FULL_SPLIT>, 4, 3> RefGpuTimeslice;  // the Coulomb apps' memory pattern

template <class FT, class MP = RefGpu>
static int load_save(const char *in, const char *out, int reinterpret, double *U, const double *Unew)
{
    LinkFile<FT, RefStandard, MP, SiteCoord<4, FULL_SPLIT>> lf((ReinterpretReal)reinterpret);
    SiteCoord<4, FULL_SPLIT> s(HOST_CONSTANTS::SIZE);
    if (!lf.load(s, in, (Real *)U)) return 1;
    if (out) {
        std::vector<double> tmp(Unew, Unew + 72 * (size_t)Nt * Nx * Ny * Nz);
        if (!lf.save(s, out, (Real *)tmp.data())) return 2;
    }
    return 0;
}

extern "C" {

void refio_size(int32_t size[4])
{
    for (int i = 0; i < 4; i++) size[i] = HOST_CONSTANTS::SIZE[i];
}

/* format 0 = PLAIN, 1 = HEADERONLY, 2 = VOGT; reinterpret 0 = STANDARD (Real = double here),
 * 1 = DOUBLE, 2 = FLOAT.  Loads `in` into U (GpuPattern, doubles); if `out` is given, the same
 * LinkFile object (its header state) then saves Unew to `out`. */
int refio_linkfile(int format, const char *in, const char *out, int reinterpret, double *U, const double *Unew)
{
    std::ostringstream sink;
    std::streambuf *old = std::cout.rdbuf(sink.rdbuf());  // the reference prints while loading
    int rc = 3;
    if (format == 0) rc = load_save<FilePlain>(in, out, reinterpret, U, Unew);
    if (format == 1) rc = load_save<FileHeaderOnly>(in, out, reinterpret, U, Unew);
    if (format == 2) rc = load_save<FileVogt>(in, out, reinterpret, U, Unew);
    std::cout.rdbuf(old);
    return rc;
}

/* the same with the memory pattern of the Coulomb apps (CoulombGaugeFixingSU3_4D.cu:57-59,132-134) */
int refio_linkfile_timeslice(int format, const char *in, const char *out, int reinterpret, double *U,
                             const double *Unew)
{
    std::ostringstream sink;
    std::streambuf *old = std::cout.rdbuf(sink.rdbuf());
    int rc = 3;
    if (format == 0) rc = load_save<FilePlain, RefGpuTimeslice>(in, out, reinterpret, U, Unew);
    if (format == 1) rc = load_save<FileHeaderOnly, RefGpuTimeslice>(in, out, reinterpret, U, Unew);
    if (format == 2) rc = load_save<FileVogt, RefGpuTimeslice>(in, out, reinterpret, U, Unew);
    std::cout.rdbuf(old);
    return rc;
}

int refio_read_ildg_timeslice(const char *path, double *U)
{
    SiteCoord<4, FULL_SPLIT> s(HOST_CONSTANTS::SIZE);
    const short size[4] = {(short)Nt, (short)Nx, (short)Ny, (short)Nz};
    readILDG_timeslice(s, path, size, (Real *)U);
    return 0;
}

int refio_write_ildg_timeslice(const char *template_path, const char *out, double *U, int steps)
{
    SiteCoord<4, FULL_SPLIT> s(HOST_CONSTANTS::SIZE);
    const short size[4] = {(short)Nt, (short)Nx, (short)Ny, (short)Nz};
    writeILDG_timeslice(s, template_path, out, size, (Real *)U, steps);
    return 0;
}

int refio_read_qcdstag_timeslice(const char *path, double *U)
{
    SiteCoord<4, FULL_SPLIT> s(HOST_CONSTANTS::SIZE);
    const short size[4] = {(short)Nt, (short)Nx, (short)Ny, (short)Nz};
    std::ostringstream sink;
    std::streambuf *old = std::cout.rdbuf(sink.rdbuf());
    const bool ok = readQCDSTAG_timeslice(s, path, size, (Real *)U);
    std::cout.rdbuf(old);
    return ok ? 0 : 1;
}

int refio_write_qcdstag_timeslice(const char *out, double *U)
{
    SiteCoord<4, FULL_SPLIT> s(HOST_CONSTANTS::SIZE);
    const short size[4] = {(short)Nt, (short)Nx, (short)Ny, (short)Nz};
    return writeQCDSTAG_timeslice(s, out, size, (Real *)U) ? 0 : 1;
}

int refio_read_ildg(const char *path, double *U)
{
    SiteCoord<4, FULL_SPLIT> s(HOST_CONSTANTS::SIZE);
    const short size[4] = {(short)Nt, (short)Nx, (short)Ny, (short)Nz};
    readILDG(s, path, size, (Real *)U);
    return 0;
}

int refio_write_ildg(const char *template_path, const char *out, double *U, int steps)
{
    SiteCoord<4, FULL_SPLIT> s(HOST_CONSTANTS::SIZE);
    const short size[4] = {(short)Nt, (short)Nx, (short)Ny, (short)Nz};
    writeILDG(s, template_path, out, size, (Real *)U, steps);
    return 0;
}

int refio_read_qcdstag(const char *path, double *U)
{
    SiteCoord<4, FULL_SPLIT> s(HOST_CONSTANTS::SIZE);
    const short size[4] = {(short)Nt, (short)Nx, (short)Ny, (short)Nz};
    std::ostringstream sink;
    std::streambuf *old = std::cout.rdbuf(sink.rdbuf());
    const bool ok = readQCDSTAG(s, path, size, (Real *)U);
    std::cout.rdbuf(old);
    return ok ? 0 : 1;
}

int refio_write_qcdstag(const char *out, double *U)
{
    SiteCoord<4, FULL_SPLIT> s(HOST_CONSTANTS::SIZE);
    const short size[4] = {(short)Nt, (short)Nx, (short)Ny, (short)Nz};
    return writeQCDSTAG(s, out, size, (Real *)U) ? 0 : 1;
}

}  // extern "C"
