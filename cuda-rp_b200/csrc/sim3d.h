// The 3-D Cartesian simulation (sim3d.cu) as seen by the C ABI in sim.cu.
#pragma once
#include <string>
#include <vector>

#include "crp.h"

namespace crp {

struct Sim3Impl;

crp_status sim3_create(const crp_config* cfg, const crp_bubbles_in* bubbles, void* stream, Sim3Impl** out,
                       std::string* err);
void sim3_destroy(Sim3Impl* s);
crp_status sim3_step(Sim3Impl* s, int n);
crp_status sim3_read_field(Sim3Impl* s, crp_field w, double* host);
crp_status sim3_read_bubbles(Sim3Impl* s, crp_bubble_field w, double* host);
crp_status sim3_set_elements(Sim3Impl* s, int n, const double* amp, const double* phase);
void sim3_dims(const Sim3Impl* s, crp_dims3* d);
const crp_stats& sim3_stats(const Sim3Impl* s);
const char* sim3_error(const Sim3Impl* s);
crp_status sim3_set_profiling(Sim3Impl* s, int on);
void* sim3_stream(Sim3Impl* s);
int sim3_device(const Sim3Impl* s);
size_t sim3_state_bytes(const Sim3Impl* s);
crp_status sim3_save_state(Sim3Impl* s, void* blob, std::vector<unsigned char>& host);
crp_status sim3_load_state(Sim3Impl* s, const void* blob, const std::vector<unsigned char>& host);
crp_status sim3_set_tuning(Sim3Impl* s, const crp_tuning* t);
void sim3_get_tuning(const Sim3Impl* s, crp_tuning* t);
crp_status sim3_adjoint(Sim3Impl* s, const crp_objective* obj, double* J, double* grad_amp, double* grad_phase);

}  // namespace crp
