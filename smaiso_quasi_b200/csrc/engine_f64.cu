// FP64 (plain form) instantiation of the engine.
#include "engine_impl.cuh"

namespace quasi {
EngineBase* make_engine_f64(const quasi_config& cfg, std::string& err) { return make_engine<double>(cfg, err); }
}  // namespace quasi
