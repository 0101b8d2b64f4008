// The reference's host-side singular correction (assembly.cu:208-321) is
// file-local (static), so this translation unit includes that source file
// from the reference tree, as it lies, and adds one C entry point that calls
// it on the mesh and RWG of ref_host_shim.cpp.  Compiled by oracle/Makefile
// into oracle/_ref/libref_host.so.  TEST INFRASTRUCTURE ONLY.
#include "assembly.cu"

const Mesh& ref_current_mesh();
const RWG& ref_current_rwg();

// L (N x N complex, row-major, as interleaved doubles) += the same-triangle
// corrections for wavenumber k and quadrature order quad_order.
extern "C" void ref_singular_corrections(int quad_order, double k_re, double k_im, double* L) {
    const RWG& r = ref_current_rwg();
    const TriQuad q = tri_quadrature(quad_order);
    apply_singular_corrections(r, ref_current_mesh(), q, std::complex<double>(k_re, k_im),
                               reinterpret_cast<std::complex<double>*>(L), r.N);
}
