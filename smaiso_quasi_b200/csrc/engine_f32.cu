// FP32 form: fields and transforms in float, constants/update/reductions in double.
#include "engine_impl.cuh"

namespace quasi {
EngineBase* make_engine_f32(const quasi_config& cfg, std::string& err) { return make_engine<float>(cfg, err); }
}  // namespace quasi
