// Oracle build support (test infrastructure, not shipped): a single-rank
// stand-in for the MPI wrapper classes declared in Bslib/ExchangeMPI.h:68-264,
// so that the reference Bslib links and runs its serial/nproc==1 code paths
// without an MPI library.  Every collective over one rank is an identity copy;
// point-to-point traffic cannot occur with one rank and aborts if reached.
// METIS entry points are aborting stubs: the oracle always runs with
// natural ordering (ordtype = 0), which never calls them.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <chrono>
#include "ExchangeMPI.h"

static void single_rank_unreachable(const char *what) {
	std::fprintf(stderr, "oracle single-rank stub: %s is not available without MPI\n", what);
	std::abort();
}

CMPIComm::CMPIComm() : comm(nullptr), ref(nullptr), procIndex(0), procGroup(0), procNumber(1) {}
CMPIComm::CMPIComm(const CMPIComm &o) : comm(o.comm), ref(nullptr), procIndex(o.procIndex), procGroup(o.procGroup), procNumber(o.procNumber) {}
CMPIComm::~CMPIComm() {}
CMPIComm &CMPIComm::operator=(const CMPIComm &o) {
	comm = o.comm; procIndex = o.procIndex; procGroup = o.procGroup; procNumber = o.procNumber;
	return *this;
}
void CMPIComm::SetCommMPI(void *c) { comm = c; procIndex = 0; procNumber = 1; }
CMPIComm CMPIComm::CreateComm(int nproc, int *) {
	if (nproc != 1) single_rank_unreachable("CMPIComm::CreateComm(nproc>1)");
	return *this;
}

CMPIRequest::CMPIRequest() : req(nullptr) {}
CMPIRequest::~CMPIRequest() {}
CMPIRequest &CMPIRequest::operator=(const CMPIRequest &o) { req = o.req; return *this; }
CMPIStatus::CMPIStatus() : stat(nullptr) {}
CMPIStatus::~CMPIStatus() {}

static size_t single_rank_type_size(MPIExchangeDataType t) {
	switch (t) {
	case CHARVALUE: case UNSIGNEDCHARVALUE: return 1;
	case SHORTVALUE: case UNSIGNEDSHORTVALUE: return 2;
	case INTEGERVALUE: case UNSIGNEDINTEGERVALUE: case FLOATVALUE: return 4;
	case DOUBLEVALUE: return 8;
	}
	return 8;
}

int CMPIExchange::ExchangeArrayMPI(const CMPIComm &, MPIExchangeDataType t, MPIExchangeOperation,
                                   int len, void *ini, void *fin) {
	if (len > 0 && ini != fin) std::memmove(fin, ini, (size_t)len * single_rank_type_size(t));
	return 0;
}
int CMPIExchange::SynchronizeMPI(const CMPIComm &) { return 0; }
int CMPIExchange::GetMyidMPIGlobal() { return 0; }
int CMPIExchange::GetNprocMPIGlobal() { return 1; }
double CMPIExchange::WallTimeMPI() {
	using namespace std::chrono;
	return duration<double>(steady_clock::now().time_since_epoch()).count();
}
int CMPIExchange::DataExchangeMPI(CMPIComm &, int nsend, int *tsend, int *isend, int *csend, int *ssend, char **osend,
                                  int &nrecv, int *&trecv, int *&irecv, int *&crecv, int *&srecv, char **&orecv) {
	// With one rank every object is addressed to rank 0: hand the send list back.
	nrecv = nsend;
	trecv = new int[nsend > 0 ? nsend : 1];
	irecv = new int[nsend > 0 ? nsend : 1];
	crecv = new int[nsend > 0 ? nsend : 1];
	srecv = new int[nsend > 0 ? nsend : 1];
	orecv = new char *[nsend > 0 ? nsend : 1];
	for (int i = 0; i < nsend; i++) {
		trecv[i] = tsend[i]; irecv[i] = isend[i]; crecv[i] = 0; srecv[i] = ssend[i];
		orecv[i] = new char[ssend[i] > 0 ? ssend[i] : 1];
		if (ssend[i] > 0) std::memcpy(orecv[i], osend[i], (size_t)ssend[i]);
	}
	(void)csend;
	return 0;
}
int CMPIExchange::GetSource(CMPIStatus &, int &s) { s = 0; return 0; }
int CMPIExchange::GetTag(CMPIStatus &, int &t) { t = 0; return 0; }
int CMPIExchange::Send(CMPIComm &, int, int, int, char *) { single_rank_unreachable("Send"); return 0; }
int CMPIExchange::ISend(CMPIComm &, int, int, int, char *, CMPIRequest &) { single_rank_unreachable("ISend"); return 0; }
int CMPIExchange::Recv(CMPIComm &, int, int, int, char *, CMPIStatus &) { single_rank_unreachable("Recv"); return 0; }
int CMPIExchange::IRecv(CMPIComm &, int, int, int, char *, CMPIRequest &) { single_rank_unreachable("IRecv"); return 0; }
int CMPIExchange::WaitAll(int n, CMPIRequest *, CMPIStatus *) { if (n > 0) single_rank_unreachable("WaitAll"); return 0; }
int CMPIExchange::WaitAny(int n, CMPIRequest *, int &, CMPIStatus &) { if (n > 0) single_rank_unreachable("WaitAny"); return 0; }
int CMPIExchange::WaitSome(int n, CMPIRequest *, int &nc, int *, CMPIStatus *) { nc = 0; if (n > 0) single_rank_unreachable("WaitSome"); return 0; }
int CMPIExchange::Test(CMPIRequest &, bool &f, CMPIStatus &) { f = true; return 0; }
int CMPIExchange::TestSome(int n, CMPIRequest *, int &nc, int *, CMPIStatus *) { nc = 0; if (n > 0) single_rank_unreachable("TestSome"); return 0; }

void CParMETIS::PartKway(CMPIComm &, int *, int *, int *, int *, int *, int *, int *, int *, int *, float *, float *,
                         int *, int *, int *) { single_rank_unreachable("ParMETIS PartKway"); }

extern "C" {
void METIS_NodeND() { single_rank_unreachable("METIS_NodeND"); }
void METIS_PartGraphKway() { single_rank_unreachable("METIS_PartGraphKway"); }
void METIS_PartGraphRecursive() { single_rank_unreachable("METIS_PartGraphRecursive"); }
void METIS_WPartGraphRecursive() { single_rank_unreachable("METIS_WPartGraphRecursive"); }
}
