// TEST INFRASTRUCTURE ONLY: link stubs for QUICK's own CUDA get2e harness.
//
// QUICK's GPU host code (src/gpu/cuda/gpu.cu) refers to the DFT exchange-
// correlation, one-electron, electrostatic-property and libxc entry points of
// other translation units.  The closed-shell Fock build (gpu_get_cshell_eri_ ->
// get2e, src/gpu/gpu_get2e_getxc_drivers.h:24-123) calls none of them, so the
// harness links these stand-ins instead of building those units.  Each one stops
// the process (host side) if it is ever reached, so a harness that drifted onto
// another path fails loudly instead of returning wrong numbers.
#include <cstdio>
#include <cstdlib>

struct gpu_type;

[[noreturn]] static void unreachable(const char* name) {
    std::fprintf(stderr, "refgpu harness: %s is outside the get2e path and is not linked\n", name);
    std::abort();
}

void getxc(gpu_type*) { unreachable("getxc"); }
void getxc_grad(gpu_type*) { unreachable("getxc_grad"); }
void get_ssw(gpu_type*) { unreachable("get_ssw"); }
void getOEI(gpu_type*) { unreachable("getOEI"); }
void get_oei_grad(gpu_type*) { unreachable("get_oei_grad"); }
void getOEPROP(gpu_type*) { unreachable("getOEPROP"); }
void get_primf_contraf_lists(gpu_type*, unsigned char*, unsigned int*, unsigned int*) {
    unreachable("get_primf_contraf_lists");
}
void upload_sim_to_constant_dft(gpu_type*) { unreachable("upload_sim_to_constant_dft"); }
void upload_sim_to_constant_oei(gpu_type*) { unreachable("upload_sim_to_constant_oei"); }
void upload_sim_to_constant_oeprop(gpu_type*) { unreachable("upload_sim_to_constant_oeprop"); }
void upload_para_to_const_oei() { unreachable("upload_para_to_const_oei"); }
void upload_para_to_const_oeprop() { unreachable("upload_para_to_const_oeprop"); }

extern "C" {
void get_gpu_work_params() { unreachable("get_gpu_work_params"); }
int xc_func_init(void*, int, int) { unreachable("xc_func_init"); }
void xc_func_end(void*) { unreachable("xc_func_end"); }
}
