// Test infrastructure only: the reference's own .tns reader (readTensor, mtxTnsIO.cpp:30-65,
// pigo) compiled from its sources, exposed with a C ABI so the tests can compare the library's
// GPU reader with it.
#include <cstdint>
#include <cstdlib>
#include <string>

#include "mtxTnsIO.hpp"

extern "C" {

int ref_read_tns(const char* path, uint32_t* d, uint32_t* n, uint32_t** idx, uint32_t** dims, double** vals) {
    unsigned dd = 0, nn = 0;
    unsigned *h = nullptr, *dm = nullptr;
    double* v = nullptr;
    readTensor(std::string(path), &h, &dm, &v, dd, nn);
    *d = dd;
    *n = nn;
    *idx = h;
    *dims = dm;
    *vals = v;
    return 0;
}

void ref_io_free(void* p) { std::free(p); }

}  // extern "C"
