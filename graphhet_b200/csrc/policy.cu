// Policy hooks; the network itself lives in mlp.cu.
#include "policy.cuh"

namespace ghb {

int policy_pick_direction(const float* /*features*/) { return -1; }
double policy_pick_delta(const float* /*features*/, double /*base_delta*/) { return -1.0; }

}  // namespace ghb
