// C++ drop-in façade over the C ABI (opendba_b200.h): the reference's
// templated host entry points for the hot path, with the reference's
// signatures, argument meaning, side effects on the caller's arrays, output
// files and process exit codes.  Instantiated for float and double in
// libopendba_b200.so.
//
//   setupAndRun<T>               openDBA.cuh:13-15
//   performDBA<T>                dba.hpp:863-864
//   approximateMedoidIndices<T>  dba.hpp:36-37
//   DBAUpdate<T>                 dba.hpp:432-434
//   normalizeSequences<T>        gpu_utils.hpp:132-133
//   adaptive_segmentation<T>     segmentation.hpp:340-343
//
// Pointers to series may be host, pinned, managed or device memory: the
// façade reads them with cudaMemcpy* (cudaMemcpyDefault).  Unlike the
// reference, no function here requires managed memory.
#ifndef OPENDBA_B200_HPP
#define OPENDBA_B200_HPP

#include <cuda_runtime.h>

#include <cstddef>
#include <string>

#include "opendba_b200.h"

// Algorithm modes of performDBA (dba.hpp:30-32).
#ifndef CLUSTER_ONLY
#define CLUSTER_ONLY 1
#define CONSENSUS_ONLY 2
#define CLUSTER_AND_CONSENSUS 3
#endif

// Input read modes (read_mode_codes.h:4-12).
#ifndef TEXT_READ_MODE
#define TEXT_READ_MODE 0
#define BINARY_READ_MODE 1
#define TSV_READ_MODE 2
#endif

// Process exit codes the reference's host code uses (exit_codes.hpp:4-32).
namespace odba_exit {
enum : int {
  CANNOT_WRITE_DISTANCE_MATRIX = 18,
  CANNOT_WRITE_DTW_PATH = 22,
  CANNOT_WRITE_DBA_AVG = 23,
  CANNOT_READ_SEQUENCE_PREFIX_FILE = 24,
  CANNOT_WRITE_DTW_PATH_MATRIX = 26,
  NOT_ENOUGH_SEQUENCES = 32,
  CANNOT_WRITE_MEMBERSHIP = 33,
  CANNOT_ALLOCATE_PAIRWISE_DIST_ARRAY = 34,
  MEMCPY_FAILURE = 35,
  MEDOID_FINDING_ERROR = 36,
  UNKNOWN_ALGO = 42,
  CANNOT_READ_MEMBERSHIP = 43,
  MEMBERSHIP_FILE_FORMAT_VIOLATION = 44,
  CANNOT_READ_DBA_AVG = 45,
  AVG_FILE_FORMAT_VIOLATION = 46,
  // not in the reference: a status from the device library (message on stderr)
  DEVICE_LIBRARY_ERROR = 60
};
}

template <typename T>
void setupAndRun(char *seqprefix_file_name, char **series_file_names, int num_series,
                 char *output_prefix, int read_mode, int use_open_start, int use_open_end,
                 char *min_segment_length_string, int norm_sequences, double cdist,
                 const int prefix_start = 0, const int prefix_length = 0, bool is_short = false);

template <typename T>
void performDBA(T **sequences, int num_sequences, size_t *sequence_lengths, char **sequence_names,
                int use_open_start, int use_open_end, char *output_prefix, int norm_sequences,
                double cdist, char **series_file_names, int num_series, int read_mode,
                bool is_segmented, int algo_mode, cudaStream_t stream = 0);

template <typename T>
int *approximateMedoidIndices(T *gpu_sequences, size_t maxSeqLength, size_t num_sequences,
                              size_t *sequence_lengths, char **sequence_names, int use_open_start,
                              int use_open_end, char *output_prefix, double *cdist,
                              int *memberships, cudaStream_t stream);

template <typename T>
double DBAUpdate(T *C, size_t centerLength, T **sequences, char **sequence_names,
                 size_t num_sequences, size_t *sequence_lengths, int use_open_start,
                 int use_open_end, T *updatedMean, std::string output_prefix, cudaStream_t stream);

template <typename T>
void normalizeSequences(T **sequences, size_t num_sequences, size_t *sequence_lengths,
                        int refSequenceIndex, double *sequence_means, double *sequence_sigmas,
                        cudaStream_t stream);

// chopPrefixFromSequences<T> (dba.hpp:1193): aligns every series to the
// leader with open-end DTW, writes <output_prefix>.prefix_chop.txt and replaces
// each series by its tail from the chop position (empty ones are dropped).
template <typename T>
void chopPrefixFromSequences(T *sequence_prefix, size_t sequence_prefix_length, T **sequences,
                             int *num_sequences, size_t *sequence_lengths, char **sequence_names,
                             char *output_prefix, int norm_sequences, cudaStream_t stream = 0);

template <typename T>
void adaptive_segmentation(T **sequences, size_t *seq_lengths, int num_seqs, int min_segment_length,
                           T ***segmented_sequences, size_t **segmented_seq_lengths,
                           int prefix_length_to_skip, cudaStream_t stream = 0);

#define ODBA_EXTERN_TEMPLATES(T)                                                               \
  extern template void chopPrefixFromSequences<T>(T *, size_t, T **, int *, size_t *, char **,   \
                                                  char *, int, cudaStream_t);                    \
  extern template void setupAndRun<T>(char *, char **, int, char *, int, int, int, char *, int, \
                                      double, const int, const int, bool);                     \
  extern template void performDBA<T>(T **, int, size_t *, char **, int, int, char *, int,       \
                                     double, char **, int, int, bool, int, cudaStream_t);       \
  extern template int *approximateMedoidIndices<T>(T *, size_t, size_t, size_t *, char **, int, \
                                                   int, char *, double *, int *, cudaStream_t); \
  extern template double DBAUpdate<T>(T *, size_t, T **, char **, size_t, size_t *, int, int,   \
                                      T *, std::string, cudaStream_t);                          \
  extern template void normalizeSequences<T>(T **, size_t, size_t *, int, double *, double *,   \
                                             cudaStream_t);                                     \
  extern template void adaptive_segmentation<T>(T **, size_t *, int, int, T ***, size_t **, int, \
                                                cudaStream_t);
ODBA_EXTERN_TEMPLATES(float)
ODBA_EXTERN_TEMPLATES(double)
#undef ODBA_EXTERN_TEMPLATES

#endif  // OPENDBA_B200_HPP
