// Test scaffolding for the oracle build only (not product code).
// Minimal stand-in for the Boost.Random names that the reference's core/RandomGenerator.h
// names: boost::mt19937, boost::normal_distribution<>, boost::variate_generator<>.
// Backed by the standard library; enough for the header to compile. The oracle never draws
// random numbers through RandomGenerator: test inputs are generated by the callers.
#ifndef ORACLE_STANDIN_BOOST_RANDOM_HPP
#define ORACLE_STANDIN_BOOST_RANDOM_HPP
#include <random>
namespace boost {
typedef std::mt19937 mt19937;
template <class T = double> class normal_distribution : public std::normal_distribution<T> {
public:
    normal_distribution(T mean = 0, T sd = 1) : std::normal_distribution<T>(mean, sd) {}
};
template <class Engine, class Dist> class variate_generator {
    Engine eng_;
    Dist dist_;
public:
    variate_generator(Engine e, Dist d) : eng_(e), dist_(d) {}
    typename Dist::result_type operator()() { return dist_(eng_); }
};
}  // namespace boost
#endif
