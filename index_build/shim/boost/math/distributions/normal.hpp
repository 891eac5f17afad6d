// Stand-in for boost::math::normal_distribution. Boost is not in this image.
// Only the distance prober names it, and that prober is never run by the
// index builder or the query oracle; calling quantile() here throws.
#pragma once
#include <stdexcept>

namespace boost {
namespace math {
template <typename RealType = double>
class normal_distribution {
public:
    normal_distribution(RealType mean = 0, RealType sd = 1) : _mean(mean), _sd(sd) {}
private:
    RealType _mean;
    RealType _sd;
};
template <typename RealType>
RealType quantile(const normal_distribution<RealType>&, RealType) {
    throw std::logic_error("boost::math::quantile is not available in this build");
}
}  // namespace math
}  // namespace boost
