// Oracle build support (test infrastructure, not shipped): the reference's
// CSMatrixR::ConvertToBinary (Bslib/smatrixr.cpp:4010) as a command-line
// program, `ref_convert <text file> <binary file>`: a matrix in the text form
// of CSMatrixR::ReadMtr followed by the right-hand side and the norm vector
// in the text form of CSVector::ReadVect, rewritten in the binary forms of
// WriteMtrBin / WriteVectBin.  It runs as its own process because the
// reference's text streams crash when its library is loaded into a Python
// process.
#include <fstream>
#include <iostream>
#include "smatrix.h"

int main(int argc, char **argv) {
	if (argc != 3) {
		std::cerr << "usage: ref_convert <text file> <binary file>\n";
		return 2;
	}
	std::ifstream fin(argv[1]);
	std::ofstream fout(argv[2], std::ios::binary | std::ios::trunc);
	std::cout.setstate(std::ios::badbit);
	try {
		CSMatrixR::ConvertToBinary(fin, fout);
	} catch (const char *e) {
		std::cerr << "ref_convert: " << e << "\n";
		return 1;
	}
	return 0;
}
