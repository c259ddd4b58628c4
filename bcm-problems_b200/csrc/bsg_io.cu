// Matrix and vector files in the reference's formats (host code).
//
// * CSMatrixR binary form, CSMatrixR::WriteMtrBin / ReadMtrBin
//   (Bslib/smatrixr.cpp:3984 / :3852): int m, n, nlist, nzja; int list[nlist],
//   ia[nlist + 1], ja[nzja]; double a[nzja] -- raw, native byte order, no
//   padding (OutArrAccV / ReadArrAccV, Bslib/globals.cpp:2209-2306).
// * CSMatrixR text form read by CSMatrixR::ReadMtr (Bslib/smatrixr.cpp:3888):
//   n and nzja as numbers, then the rest of that line and a label line are
//   skipped, ia[n + 1]; the rest of the line and a label line, ja[nzja]; the
//   rest of the line and a label line, a[nzja].  list = 0 .. n - 1.
// * CSVector text form read by CSVector::ReadVect (Bslib/svector.cpp:465): the
//   rest of the current line and a label line are skipped, then nv numbers
//   (ConvertToBinary, Bslib/smatrixr.cpp:4010, reads a matrix and then the
//   right-hand side and the norm vector this way from one file).
// * CSVector binary form, CSVector::WriteVectBin / ReadVectBin
//   (Bslib/svector.cpp:537 / :488): int nparts, nrhs, nv; double v[nv * nrhs];
//   int blksv[nparts + 1], inda[nparts].
//
// Every reader works at a byte offset of the file and, when it has filled the
// arrays, moves the offset past what it read, so the pieces of one file (a
// matrix followed by vectors) are read one after another, as the reference
// reads them from one stream.  Called with NULL arrays a reader returns the
// sizes only and leaves the offset alone.
#include "bsg_internal.cuh"
#include <cstdio>
#include <fstream>
#include <limits>
#include <string>
#include <vector>

namespace {

// Sizes written by the reference are int; a negative size or one that does
// not fit the file is a malformed file.
int bad(const char *what, const char *path) {
	char msg[512];
	std::snprintf(msg, sizeof msg, "%s: malformed or truncated file %s", what, path ? path : "(null)");
	return bsg_set_error(BSG_ERR_ARG, msg);
}

template <class T>
bool rd(std::ifstream &f, T *p, long long count) {
	if (count < 0) return false;
	if (count == 0) return true;
	if (!p) {
		f.seekg((std::streamoff)(sizeof(T) * count), std::ios::cur);
		return (bool)f;
	}
	f.read(reinterpret_cast<char *>(p), (std::streamsize)(sizeof(T) * count));
	return f.gcount() == (std::streamsize)(sizeof(T) * count);
}

template <class T>
bool wr(std::ofstream &f, const T *p, long long count) {
	if (count <= 0) return true;
	if (!p) return false;
	f.write(reinterpret_cast<const char *>(p), (std::streamsize)(sizeof(T) * count));
	return (bool)f;
}

bool open_in(std::ifstream &f, const char *path, const long long *offset) {
	if (!path || !offset || *offset < 0) return false;
	f.open(path, std::ios::binary);
	if (!f) return false;
	f.seekg((std::streamoff)*offset);
	return (bool)f;
}

bool open_out(std::ofstream &f, const char *path, int append) {
	if (!path) return false;
	f.open(path, std::ios::binary | (append ? std::ios::app : std::ios::trunc));
	return (bool)f;
}

// getline with the reference's 10-byte buffer semantics is only used to skip
// the rest of a line and short label lines; skipping whole lines is the same
// on every file the reference itself can read.
void skip_line(std::ifstream &f) { f.ignore(std::numeric_limits<std::streamsize>::max(), '\n'); }

// Byte position after a successful read; a read that ended exactly at the end
// of the file leaves eofbit set, which tellg() would turn into a failure.
long long pos_after(std::ifstream &f) {
	f.clear();
	return (long long)f.tellg();
}

} // namespace

extern "C" int bsg_read_mtr_bin(const char *path, long long *offset, int *m, int *n, int *nlist, int *nzja, int *list,
                                int *ia, int *ja, double *a) {
	std::ifstream f;
	if (!open_in(f, path, offset)) return bad("bsg_read_mtr_bin", path);
	int hdr[4];
	if (!rd(f, hdr, 4) || hdr[2] < 0 || hdr[3] < 0) return bad("bsg_read_mtr_bin", path);
	if (m) *m = hdr[0];
	if (n) *n = hdr[1];
	if (nlist) *nlist = hdr[2];
	if (nzja) *nzja = hdr[3];
	if (!list && !ia && !ja && !a) return BSG_OK;
	if (!list || !ia || (hdr[3] > 0 && (!ja || !a))) return bsg_set_error(BSG_ERR_ARG, "bsg_read_mtr_bin: null array");
	if (!rd(f, list, hdr[2]) || !rd(f, ia, (long long)hdr[2] + 1) || !rd(f, ja, hdr[3]) || !rd(f, a, hdr[3]))
		return bad("bsg_read_mtr_bin", path);
	if (ia[hdr[2]] != hdr[3]) return bad("bsg_read_mtr_bin (ia[nlist] != nzja)", path);
	*offset = pos_after(f);
	return BSG_OK;
}

extern "C" int bsg_write_mtr_bin(const char *path, int append, int m, int n, int nlist, const int *list, const int *ia,
                                 const int *ja, const double *a) {
	if (nlist < 0 || !ia || !list) return bsg_set_error(BSG_ERR_ARG, "bsg_write_mtr_bin: bad argument");
	std::ofstream f;
	if (!open_out(f, path, append)) return bsg_set_error(BSG_ERR_ARG, "bsg_write_mtr_bin: cannot open the file");
	const int nz = ia[nlist];
	const int hdr[4] = {m, n, nlist, nz};
	if (!wr(f, hdr, 4) || !wr(f, list, nlist) || !wr(f, ia, (long long)nlist + 1) || !wr(f, ja, nz) || !wr(f, a, nz))
		return bsg_set_error(BSG_ERR_ARG, "bsg_write_mtr_bin: write failed");
	return BSG_OK;
}

extern "C" int bsg_read_mtr(const char *path, long long *offset, int *n, int *nzja, int *ia, int *ja, double *a) {
	std::ifstream f;
	if (!open_in(f, path, offset)) return bad("bsg_read_mtr", path);
	long long nl = -1, nz = -1;
	f >> nl >> nz;
	if (!f || nl < 0 || nz < 0 || nl > 0x7fffffffLL - 1 || nz > 0x7fffffffLL) return bad("bsg_read_mtr", path);
	if (n) *n = (int)nl;
	if (nzja) *nzja = (int)nz;
	if (!ia && !ja && !a) return BSG_OK;
	if (!ia || (nz > 0 && (!ja || !a))) return bsg_set_error(BSG_ERR_ARG, "bsg_read_mtr: null array");
	skip_line(f);
	skip_line(f);
	for (long long i = 0; i <= nl; i++) f >> ia[i];
	skip_line(f);
	skip_line(f);
	for (long long i = 0; i < nz; i++) f >> ja[i];
	skip_line(f);
	skip_line(f);
	for (long long i = 0; i < nz; i++) f >> a[i];
	if (f.fail()) return bad("bsg_read_mtr", path);
	*offset = pos_after(f);
	return BSG_OK;
}

extern "C" int bsg_read_vect(const char *path, long long *offset, int nv, double *v) {
	std::ifstream f;
	if (nv < 0 || (nv > 0 && !v)) return bsg_set_error(BSG_ERR_ARG, "bsg_read_vect: bad argument");
	if (!open_in(f, path, offset)) return bad("bsg_read_vect", path);
	skip_line(f);
	skip_line(f);
	for (int i = 0; i < nv; i++) f >> v[i];
	if (f.fail()) return bad("bsg_read_vect", path);
	*offset = pos_after(f);
	return BSG_OK;
}

extern "C" int bsg_write_vect_bin(const char *path, int append, int nv, int nrhs, int nparts, const double *v,
                                  const int *blksv, const int *inda) {
	if (nv < 0 || nrhs < 0 || nparts < 0 || (nv > 0 && nrhs > 0 && !v) || !blksv || (nparts > 0 && !inda))
		return bsg_set_error(BSG_ERR_ARG, "bsg_write_vect_bin: bad argument");
	std::ofstream f;
	if (!open_out(f, path, append)) return bsg_set_error(BSG_ERR_ARG, "bsg_write_vect_bin: cannot open the file");
	const int hdr[3] = {nparts, nrhs, nv};
	if (!wr(f, hdr, 3) || !wr(f, v, (long long)nv * nrhs) || !wr(f, blksv, (long long)nparts + 1) ||
	    !wr(f, inda, nparts))
		return bsg_set_error(BSG_ERR_ARG, "bsg_write_vect_bin: write failed");
	return BSG_OK;
}

extern "C" int bsg_read_vect_bin(const char *path, long long *offset, int *nv, int *nrhs, int *nparts, double *v,
                                 int *blksv, int *inda) {
	std::ifstream f;
	if (!open_in(f, path, offset)) return bad("bsg_read_vect_bin", path);
	int hdr[3];
	if (!rd(f, hdr, 3) || hdr[0] < 0 || hdr[1] < 0 || hdr[2] < 0) return bad("bsg_read_vect_bin", path);
	if (nparts) *nparts = hdr[0];
	if (nrhs) *nrhs = hdr[1];
	if (nv) *nv = hdr[2];
	if (!v && !blksv && !inda) return BSG_OK;
	const long long len = (long long)hdr[2] * hdr[1];
	if ((len > 0 && !v) || !blksv || (hdr[0] > 0 && !inda)) return bsg_set_error(BSG_ERR_ARG, "bsg_read_vect_bin: null array");
	if (!rd(f, v, len) || !rd(f, blksv, (long long)hdr[0] + 1) || !rd(f, inda, hdr[0]))
		return bad("bsg_read_vect_bin", path);
	*offset = pos_after(f);
	return BSG_OK;
}
