// A C++ caller written against the reference's class names (the wiring of
// nicp_simple_aligner.cpp:100-165), built with g++ against nicp.hpp and
// libnicp_b200.so.  Reads a binary file of two u16 depth frames, prints the
// pose, error and inliers.
#include <cstdio>
#include <vector>

#include "nicp_b200/nicp.hpp"

int main(int argc, char **argv) {
  if (argc < 8) {
    std::fprintf(stderr, "usage: %s frames.bin rows cols fx fy cx cy\n", argv[0]);
    return 2;
  }
  int rows = std::atoi(argv[2]), cols = std::atoi(argv[3]);
  nicp::Matrix3f K = {{(float)std::atof(argv[4]), 0, (float)std::atof(argv[6]), 0, (float)std::atof(argv[5]),
                       (float)std::atof(argv[7]), 0, 0, 1}};
  std::vector<uint16_t> buf(2 * (size_t)rows * cols);
  FILE *f = std::fopen(argv[1], "rb");
  if (!f || std::fread(buf.data(), 2, buf.size(), f) != buf.size()) return 3;
  std::fclose(f);
  try {
    nicp::PinholePointProjector proj;
    proj.setCameraMatrix(K);
    nicp::StatsCalculatorIntegralImage stats;
    nicp::PointInformationMatrixCalculator pim;
    nicp::NormalInformationMatrixCalculator nim;
    nicp::DepthImageConverterIntegralImage conv(&proj, &stats, &pim, &nim);
    nicp::Cloud ref, cur;
    conv.compute(ref, buf.data(), rows, cols);
    conv.compute(cur, buf.data() + (size_t)rows * cols, rows, cols);
    nicp::CorrespondenceFinderProjective cf;
    nicp::Linearizer lin;
    nicp::AlignerProjective aligner(&proj, &lin, &cf);
    aligner.setReferenceCloud(&ref);
    aligner.setCurrentCloud(&cur);
    aligner.setInitialGuess(nicp::Isometry3f::Identity());
    aligner.setSensorOffset(nicp::Isometry3f::Identity());
    aligner.align();
    const double *T = aligner.Td();
    for (int i = 0; i < 16; i++) std::printf("%.17g%c", T[i], i == 15 ? '\n' : ' ');
    std::printf("%.9g %d %d %zu\n", aligner.error(), aligner.inliers(), aligner.solutionValid() ? 1 : 0, ref.size());
  } catch (const nicp::Error &e) {
    std::fprintf(stderr, "nicp error %d: %s\n", e.code, e.what());
    return 1;
  }
  return 0;
}
