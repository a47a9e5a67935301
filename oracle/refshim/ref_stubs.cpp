// Definitions for symbols the reference declares but whose sources are absent
// from its tree (src/metrics/metrics.cpp and src/preprocessing/interactions.cpp
// are listed in its CMakeLists.txt but do not exist).  None is reachable with
// the options the oracle uses (early_stopping_metric="loss",
// auto_interactions=false); each throws if it is ever reached.
// Test infrastructure only.
#include <stdexcept>
#include "turbocat/interactions.hpp"
#include "turbocat/metrics.hpp"

namespace turbocat {

Float Metrics::roc_auc(const Float*, const Float*, Index) {
  throw std::runtime_error("oracle build: roc_auc source absent from the reference");
}
Float Metrics::pr_auc(const Float*, const Float*, Index) {
  throw std::runtime_error("oracle build: pr_auc source absent from the reference");
}
Float Metrics::find_optimal_threshold(const Float*, const Float*, Index, MetricType, int) {
  throw std::runtime_error("oracle build: find_optimal_threshold source absent from the reference");
}
std::vector<FeatureInteraction> InteractionDetector::detect(const Dataset&, const InteractionConfig&) {
  throw std::runtime_error("oracle build: interactions source absent from the reference");
}
FeatureIndex InteractionGenerator::generate(Dataset&, const std::vector<FeatureInteraction>&,
                                            const InteractionConfig&) {
  throw std::runtime_error("oracle build: interactions source absent from the reference");
}
void InteractionGenerator::apply(Dataset&, const Dataset&) {
  throw std::runtime_error("oracle build: interactions source absent from the reference");
}

}  // namespace turbocat
