// steppecu_b200/csrc/f2_umma.cu — placeholder until the tcgen05 contraction lands.
#include "stpf2_internal.cuh"

namespace stpf2 {

struct UmmaPlan {};

UmmaPlan* umma_plan_create(Ctx&, const OperandPlanes&, const BlockLayout&) {
    fail(STP_INVALID_CONFIG, "tcgen05 contraction not built");
}
void umma_plan_destroy(UmmaPlan* p) { delete p; }
void launch_f2_umma(Ctx&, UmmaPlan*, double*, double*, cudaStream_t) {
    fail(STP_INVALID_CONFIG, "tcgen05 contraction not built");
}
int umma_tile() { return 128; }

}  // namespace stpf2
