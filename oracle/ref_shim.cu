// ref_shim.cu -- TEST INFRASTRUCTURE ONLY.
//
// Compiled together with the reference's own CUDA sources (see
// oracle/Makefile.ref) into oracle/_ref/libdemsph_ref.so, so that tests can
// run the reference kernels on the GPU next to this library.  The reference
// sets its material tables through a C++ member function
// (contactModelParameters::buildFromTables, DEMSPH/kernel/contactKernel.cu:6-104);
// this shim exposes that one call as C so ctypes can reach it.
#include <vector>

#include "contactParameters.h"

extern "C" void ref_set_contact_tables(int nh, const double* h, int nl, const double* l, int nb, const double* b,
                                       cudaStream_t stream) {
    // rows: h = nh x (a, b, 8 values), l = nl x (a, b, 11 values), b = nb x (a, b, 6 values)
    std::vector<HertzianRow> H(nh);
    for (int k = 0; k < nh; k++) {
        const double* r = h + 10 * k;
        H[k] = HertzianRow{(int)r[0], (int)r[1], r[2], r[3], r[4], r[5], r[6], r[7], r[8], r[9]};
    }
    std::vector<LinearRow> L(nl);
    for (int k = 0; k < nl; k++) {
        const double* r = l + 13 * k;
        L[k] = LinearRow{(int)r[0], (int)r[1], r[2], r[3], r[4], r[5], r[6], r[7], r[8], r[9], r[10], r[11], r[12]};
    }
    std::vector<BondedRow> B(nb);
    for (int k = 0; k < nb; k++) {
        const double* r = b + 8 * k;
        B[k] = BondedRow{(int)r[0], (int)r[1], r[2], r[3], r[4], r[5], r[6], r[7]};
    }
    static contactModelParameters* params = nullptr;  // owns the device tables until exit
    if (!params) params = new contactModelParameters();
    params->buildFromTables(H, L, B, stream);
    cudaStreamSynchronize(stream);
}
