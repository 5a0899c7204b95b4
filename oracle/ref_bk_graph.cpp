// Builds the reference's BK 3.03 graph.cpp (benchmark/GridCut/code/BK303/graph.cpp)
// in place, adding the 64-bit flow instantiation the reference lacks
// (BK303/instances.inc:12-15 has no int64 flow type; grid max-flows exceed int32).
// TEST INFRASTRUCTURE ONLY (oracle/_ref); compiled by oracle/Makefile.
#include "graph.cpp"
template class Graph<int, int, long long>;
