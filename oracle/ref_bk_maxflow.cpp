// Builds the reference's BK 3.03 maxflow.cpp in place with the int64 flow
// instantiation (see ref_bk_graph.cpp).  TEST INFRASTRUCTURE ONLY.
#include "maxflow.cpp"
template class Graph<int, int, long long>;
