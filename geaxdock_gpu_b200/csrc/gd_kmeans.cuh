/*
 * gd_kmeans.cuh -- batched k-means of the post-Monte-Carlo clustering (gd_kmeans.cu).
 */
#ifndef GD_KMEANS_CUH
#define GD_KMEANS_CUH

#include <cstdint>
#include <string>
#include <vector>

namespace gd {

struct KmeansJob {
  const float *objects = nullptr; /* host [n][dim] */
  int dim = 9;
  std::vector<int> seg_off;       /* n_seg + 1 offsets into the objects */
  std::vector<int> k;             /* clusters per segment */
  uint64_t seed = 0;
  float threshold = 0.001f;
  int max_iter = 500;
  void *stream = nullptr;
};

struct KmeansResult {
  std::vector<int> membership;   /* [n] cluster within the segment, original object order */
  std::vector<int> medoid;       /* [clusters] representative object index, -1 if empty */
  std::vector<int> size;         /* [clusters] members */
  std::vector<int> cluster_base; /* [n_seg] first cluster of each segment */
  std::vector<int> passes;       /* [n_seg] Lloyd passes (the reference's loop_iterations) */
};

/* clusters of segment s: min(k[s], n_s); 0 on success, < 0 with err set otherwise */
int kmeans_device(const KmeansJob &job, KmeansResult &res, std::string &err);
/* the shuffle of segment `seg` of n objects: out[i] = object at shuffled position i */
int kmeans_permutation(uint64_t seed, int seg, int n, int *out);

}  // namespace gd

#endif
