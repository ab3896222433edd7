// Regenerates the seeded inputs of the reference's FFNT known-answer tests
// (test/test_fft_roundtrip.cu:145-149 and :249-253) with the same standard
// library engines and distributions, for both degrees the reference tests
// (N = 1024 and N = 2048, test/test_fft_roundtrip.cu:315-319):
//   fft_roundtrip_in.f64      1024 doubles, std::mt19937(42),
//                             uniform_real_distribution<double>(-100, 100)
//   negacyclic_random_in.i32  1024 ints,    std::mt19937(123),
//                             uniform_int_distribution<int>(-5, 5)
//   fft2_roundtrip_in.f64     the same with 2048 values
//   negacyclic2_random_in.i32 the same with 2048 values
#include <cstdio>
#include <random>
#include <vector>

static void write_inputs(const char* dir, int n, const char* fname, const char* iname)
{
    char path[4096];
    {
        std::mt19937 rng(42);
        std::uniform_real_distribution<double> dist(-100.0, 100.0);
        std::vector<double> v(n);
        for (auto& x : v) x = dist(rng);
        std::snprintf(path, sizeof(path), "%s/%s", dir, fname);
        FILE* f = std::fopen(path, "wb");
        std::fwrite(v.data(), sizeof(double), v.size(), f);
        std::fclose(f);
    }
    {
        std::mt19937 rng(123);
        std::uniform_int_distribution<int> dist(-5, 5);
        std::vector<int> v(n);
        for (auto& x : v) x = dist(rng);
        std::snprintf(path, sizeof(path), "%s/%s", dir, iname);
        FILE* f = std::fopen(path, "wb");
        std::fwrite(v.data(), sizeof(int), v.size(), f);
        std::fclose(f);
    }
}

int main(int argc, char** argv)
{
    const char* dir = argc > 1 ? argv[1] : ".";
    write_inputs(dir, 1024, "fft_roundtrip_in.f64", "negacyclic_random_in.i32");
    write_inputs(dir, 2048, "fft2_roundtrip_in.f64", "negacyclic2_random_in.i32");
    return 0;
}
