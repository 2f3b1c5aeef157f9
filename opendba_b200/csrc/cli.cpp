// openDBA command line (openDBA.cu:11-158): same positional arguments, type
// dispatch and exit codes, running the B200 library through the C++ façade.
//
//   openDBA <binary|text|tsv> <int|uint|ulong|float|double|short>
//           <global|open_start|open_end|open|open_prefix_S_L> <output prefix>
//           <minimum segment length[,for consensus]> <prefix sequence|/dev/null>
//           <clustering threshold> <series.tsv | series1 series2 ...>
//
// Integer value types are read into float, as the B200 kernels compute in
// float or double only (the reference instantiates int/uint/ulong for DTW).
#include <getopt.h>

#include <cstdlib>
#include <cstring>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "opendba.hpp"

int main(int argc, char **argv) {
  int norm_sequences = 1;
  int prefix_to_skip = 0;
  int prefix_length = 0;
  int c;
  while ((c = getopt(argc, argv, "n")) != -1) {
    switch (c) {
      case 'n':
        norm_sequences = 0;
        break;
      default:
        break;
    }
  }
  if (argc < 9) {
    std::cout << "Usage: " << argv[0] << " <binary|text|tsv> <short|int|uint|ulong|float|double> "
              << "<global|open_start|open_end|open> <output files prefix> <minimum unimodal segment "
                 "length for clustering[,for consensus generation]> <prefix sequence to "
                 "remove|/dev/null> <clustering threshold> <series.tsv|<series1> <series2> [series3...]>\n";
    std::exit(1);
  }
  const int num_series = argc - 8;
  char *min_segment_length = argv[5];
  int read_mode = TEXT_READ_MODE;
  if (!std::strcmp(argv[1], "binary")) {
    read_mode = BINARY_READ_MODE;
  } else if (!std::strcmp(argv[1], "tsv")) {
    read_mode = TSV_READ_MODE;
  } else if (std::strcmp(argv[1], "text")) {
    std::cerr << "First argument (" << argv[1] << ") is neither 'binary' nor 'text'" << std::endl;
    std::exit(1);
  }
  int use_open_start = 0, use_open_end = 0;
  if (!std::strcmp(argv[3], "global")) {
  } else if (!std::strcmp(argv[3], "open_start")) {
    use_open_start = 1;
  } else if (!std::strcmp(argv[3], "open_end")) {
    use_open_end = 1;
  } else if (!std::strncmp(argv[3], "open_prefix", 11)) {
    use_open_start = 0;
    use_open_end = 1;
    norm_sequences = 1;
    std::stringstream ss(std::string(argv[3] + 12));
    std::vector<std::string> fields;
    std::string tmp;
    while (std::getline(ss, tmp, '_')) fields.push_back(tmp);
    if (fields.size() != 2) {
      std::cerr << "Unexpected alignment type specified, expected open_prefix_##_## but did not "
                   "find a second underscore in "
                << argv[3] << std::endl;
      std::exit(1);
    }
    prefix_to_skip = std::stoi(fields[0]);
    prefix_length = std::stoi(fields[1]);
    std::cerr << "Aligning only the first " << prefix_length << " elements of each sequence" << std::endl;
  } else if (!std::strcmp(argv[3], "open")) {
    use_open_start = 1;
    use_open_end = 1;
  } else {
    std::cerr << "Third argument (" << argv[3]
              << ") is not one of the accept values 'global', 'open_start', 'open_end' or 'open'" << std::endl;
    std::exit(1);
  }
  char *output_prefix = argv[4];
  char *seqprefix_filename = nullptr;
  if (std::strcmp(argv[6], "/dev/null")) seqprefix_filename = argv[6];
  const double cdist = std::atof(argv[7]);
  const int argind = 8;
  const std::string ty = argv[2];
  if (ty == "float" || ty == "int" || ty == "uint" || ty == "ulong") {
    setupAndRun<float>(seqprefix_filename, &argv[argind], num_series, output_prefix, read_mode,
                       use_open_start, use_open_end, min_segment_length, norm_sequences, cdist,
                       prefix_to_skip, prefix_length);
  } else if (ty == "double") {
    setupAndRun<double>(seqprefix_filename, &argv[argind], num_series, output_prefix, read_mode,
                        use_open_start, use_open_end, min_segment_length, norm_sequences, cdist,
                        prefix_to_skip, prefix_length);
  } else if (ty == "short") {
    setupAndRun<float>(seqprefix_filename, &argv[argind], num_series, output_prefix, read_mode,
                       use_open_start, use_open_end, min_segment_length, norm_sequences, cdist,
                       prefix_to_skip, prefix_length, true);
  } else {
    std::cerr << "Second argument (" << argv[2]
              << ") was not one of the accepted numerical representations: 'int', 'uint', "
                 "'ulong', 'float' or 'double'"
              << std::endl;
    std::exit(1);
  }
  int devices = 0;
  cudaGetDeviceCount(&devices);
  for (int i = 0; i < devices; ++i) {
    cudaSetDevice(i);
    cudaDeviceReset();
  }
  return 0;
}
