// HogbomB200.h -- the reference's Hogbom CLEAN class (current/tHogbomCleanOMP/HogbomGolden.h,
// attic/tHogbomCleanCuda/HogbomCuda.h) on the B200 library: same deconvolve() signature and
// meaning (residual = dirty cleaned; model accumulated into), with the parameters of the
// reference's Parameters.h as defaults.  Results are bit-identical to HogbomGolden's.  Errors are
// thrown as std::runtime_error.
#ifndef TCONVOLVE_B200_HOGBOM_H
#define TCONVOLVE_B200_HOGBOM_H

#include <cstddef>
#include <vector>

class HogbomB200 {
public:
    // Parameters.h: g_niters 1000, g_gain 0.1, g_threshold 0.00001
    explicit HogbomB200(unsigned int niters = 1000, float gain = 0.1f, float threshold = 0.00001f);

    void deconvolve(const std::vector<float>& dirty, const size_t dirtyWidth, const std::vector<float>& psf,
                    const size_t psfWidth, std::vector<float>& model, std::vector<float>& residual);

    // after deconvolve: iterations carried out and the device time of the loop (s)
    int iterations() const { return done_; }
    double deviceSeconds() const { return seconds_; }

private:
    unsigned int niters_;
    float gain_, threshold_;
    int done_ = 0;
    double seconds_ = 0.0;
};

#endif
