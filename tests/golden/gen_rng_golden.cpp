// Golden vectors for the factory RNG: the exact doubles that
// std::mt19937(seed) + std::normal_distribution<double>(0,1) produce with
// libstdc++ (the generator behind the reference's StdVectorFactory /
// EigenVectorFactory). Vectors of odd length exercise the cached second
// variate of the polar method, which carries over between vectors.
// Build and run: see make_golden.py.
#include <cstdio>
#include <random>
int main() {
  const unsigned seeds[] = {1u, 42u, 7u};
  const int lens[] = {1, 3, 1000, 997, 5};
  for (unsigned s : seeds) {
    std::mt19937 gen(s);
    std::normal_distribution<double> dist(0.0, 1.0);
    std::printf("seed %u\n", s);
    for (int L : lens) {
      std::printf("vec %d\n", L);
      for (int i = 0; i < L; ++i) std::printf("%a\n", dist(gen));
    }
  }
  return 0;
}
