// ref_autostop.cpp -- C entry points to the reference's own AutoStop class
// (host/inc/autostop.hpp, compiled unchanged from the reference checkout),
// for the parity tests of the device-side AutoStop.  Test infrastructure only.
#include <string>

#include "autostop.hpp"

namespace {
struct RefAutoStop {
	std::string out;       // the class's progress table goes here, not to stdout
	AutoStop as;
	RefAutoStop(int pop, int runs, float stopstd, int asfreq) : out(), as(pop, runs, stopstd, asfreq, &out) {}
};
}  // namespace

extern "C" {

void* adgpu_ref_autostop_new(int pop_size, int num_runs, float stopstd, int as_frequency)
{
	return new RefAutoStop(pop_size, num_runs, stopstd, as_frequency);
}

// check_if_satisfactory (autostop.hpp:169-222) on the R*P current energies.
int adgpu_ref_autostop_check(void* h, int generation_cnt, const float* energies, unsigned long total_evals)
{
	return static_cast<RefAutoStop*>(h)->as.check_if_satisfactory(generation_cnt, energies, total_evals) ? 1 : 0;
}

void adgpu_ref_autostop_free(void* h) { delete static_cast<RefAutoStop*>(h); }

}  // extern "C"
