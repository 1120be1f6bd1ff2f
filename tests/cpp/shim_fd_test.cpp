// shim_fd_test.cpp -- finite-difference check of the GpuKernelEvaluator drop-in, in the manner of
// the reference's test/itkFiniteDifferenceTest.cpp (GetValue == GetValueAndDerivative value,
// then difference quotients on random parameter indices), without ITK: the images, the
// control-point grid (itkTransformAdapter.hxx:246-308 restated) and the kernel are built directly
// with the reference's own boundary types, and the moving image is prefiltered by the
// reference's BsplineImage::computeCoeffs.
//
// Exit code 0 when every check passes.  Usage: shim_fd_test [metric 0=MSE 1=NCC] [seed]
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <random>
#include <vector>

#include "skm_gpu_evaluator.hpp"

typedef Vec<ScalarType, SpaceDimensions> VecF;
typedef Vec<int, SpaceDimensions> VecI;
typedef Mat<ScalarType, SpaceDimensions> MatF;

int main(int argc, char **argv)
{
    const int metric = argc > 1 ? std::atoi(argv[1]) : 1;
    const unsigned seed = argc > 2 ? unsigned(std::atoi(argv[2])) : 7u;
    std::mt19937 rng(seed);
    std::uniform_real_distribution<double> U(0.0, 1.0);
    const int D = SpaceDimensions;
    VecI size;
    for (int d = 0; d < D; ++d) size[d] = 24 + 4 * d;
    VecF spacing(1.0), origin(0.0);
    const int N = size.product();
    // smooth images: sums of Gaussian blobs
    std::vector<ScalarType> fixed(N), moving(N);
    for (int img = 0; img < 2; ++img) {
        std::vector<ScalarType> &v = img ? moving : fixed;
        std::fill(v.begin(), v.end(), ScalarType(0));
        for (int b = 0; b < 5; ++b) {
            double c[3], s = 3.0 + 4.0 * U(rng), a = 0.3 + 0.7 * U(rng);
            for (int d = 0; d < D; ++d) c[d] = U(rng) * size[d];
            for (int i = 0; i < N; ++i) {
                int r = i;
                double q = 0;
                for (int d = 0; d < D; ++d) {
                    const int x = r % size[d];
                    r /= size[d];
                    q += (x - c[d]) * (x - c[d]);
                }
                v[i] += ScalarType(a * std::exp(-q / (2 * s * s)));
            }
        }
    }
    // moving image coefficients with the reference's prefilter
    BsplineImage<ScalarType, SpaceDimensions> movingImage(nullptr, origin, spacing, size);
    std::unique_ptr<ScalarType[]> coeffs;
    movingImage.computeCoeffs(moving.data(), coeffs);
    movingImage.assignCoeffs(coeffs.get());
    ImageNearest<ScalarType, SpaceDimensions> fixedImage(fixed.data(), origin, spacing, size);
    // control-point grid: spacing sigma, size ceil(extent/sigma), centred (itkTransformAdapter.hxx:246-308)
    const double sigmaC4 = 6.0, sigmaC0 = 12.0, cpSpacing = 2.0;
    VecI cpSize;
    VecF cpOrigin, cpScale(cpSpacing);
    for (int d = 0; d < D; ++d) {
        const double ext = (size[d] - 1) * spacing[d];
        cpSize[d] = int(std::ceil(std::abs(ext / cpSpacing)));
        cpOrigin[d] = origin[d] + std::abs(ext - (cpSize[d] - 1) * cpSpacing) / 2.0;
    }
    const int C = cpSize.product();
    ImageNearest<VecF, SpaceDimensions> cpImage(nullptr, cpOrigin, cpScale, cpSize);
    ImageNearest<ScalarType, SpaceDimensions> cpwImage(nullptr, cpOrigin, cpScale, cpSize);
    std::vector<ScalarType> w1(1, 0);
    std::vector<MatF> t1(1, MatF::identity());
    ImageNearest<ScalarType, SpaceDimensions> wimg(w1.data(), VecF(0.0), VecF(1.0), VecI(1));
    ImageNearest<MatF, SpaceDimensions> wten(t1.data(), VecF(0.0), VecF(1.0), VecI(1));
    Kernel kernel(sigmaC0, sigmaC4, false, 0.0, wimg, false, MatF::identity(), wten);

    GpuKernelEvaluator ev(C * D, 1, 1, kernel, movingImage, fixedImage, cpImage, cpwImage);
    ev.SetRegularizerRD(1e-3);
    std::vector<VecF> cp(C);
    std::vector<ScalarType> cpw(C, ScalarType(1));
    for (int i = 0; i < C; ++i)
        // U[-0.1,0.1]: displacements stay below half a voxel, so no sample crosses the moving image's
        // inside test (which makes the metric discontinuous) while the differences are taken
        for (int d = 0; d < D; ++d) cp[i][d] = ScalarType(0.2 * U(rng) - 0.1);
    const GpuKernelEvaluator::MEASURE m = metric == 0 ? GpuKernelEvaluator::MEASURE::MSE : GpuKernelEvaluator::MEASURE::NCC;
    std::vector<ScalarType> der(C * D);
    auto v1 = ev.getValue(m, cp.data(), cpw.data(), ImageNearest<VecF, SpaceDimensions>(), false);
    auto v2 = ev.getValueAndDerivative(m, cp.data(), cpw.data(), ImageNearest<VecF, SpaceDimensions>(), der.data(),
                                       false);
    int failures = 0;
    if (v1.measure != v2.measure || v1.reg_value_rd != v2.reg_value_rd) {
        std::printf("GetValue %.17g != GetValueAndDerivative %.17g\n", double(v1.measure), double(v2.measure));
        ++failures;
    }
    auto total = [&](const GpuKernelEvaluator::EvaluationResult &r) { return double(r.measure) + 1e-3 * double(r.reg_value_rd); };
    double gmax = 0;
    for (int i = 0; i < C * D; ++i) gmax = std::max(gmax, std::abs(double(der[i])));
    // central differences on the 30 largest-gradient indices and 30 random ones
    std::vector<int> idx(C * D);
    for (int i = 0; i < C * D; ++i) idx[i] = i;
    std::partial_sort(idx.begin(), idx.begin() + 30, idx.end(),
                      [&](int a, int b) { return std::abs(der[a]) > std::abs(der[b]); });
    for (int k = 0; k < 30; ++k) idx[30 + k] = int(U(rng) * (C * D - 1));
    const double h = 2e-3;
    double worst = 0;
    for (int k = 0; k < 60; ++k) {
        const int p = idx[k];
        const int cpi = p % C, d = p / C;       // planar layout [d*C + i]
        const ScalarType keep = cp[cpi][d];
        cp[cpi][d] = keep + h;
        const double fp = total(ev.getValue(m, cp.data(), cpw.data(), ImageNearest<VecF, SpaceDimensions>(), false));
        cp[cpi][d] = keep - h;
        const double fm = total(ev.getValue(m, cp.data(), cpw.data(), ImageNearest<VecF, SpaceDimensions>(), false));
        cp[cpi][d] = keep;
        const double fd = (fp - fm) / (2 * h);
        const double err = std::abs(fd - double(der[p])) / gmax;
        worst = std::max(worst, err);
    }
    std::printf("metric %d: value %.10f, |grad|max %.3e, worst |fd - grad| / |grad|max over 60 indices = %.3e\n",
                metric, double(v2.measure), gmax, worst);
    if (!(worst < 2e-2)) ++failures;
    if (!(gmax > 0)) ++failures;
    return failures ? 1 : 0;
}
