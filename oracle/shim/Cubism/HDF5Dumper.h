// Oracle test infrastructure: stand-in for Cubism's HDF5 field dumper
// (SimulationData.cpp:49-97).  HDF5 is absent on this machine; field output
// is not part of the timestep path, so every dump is a no-op here.
#pragma once
#include <string>
template <typename TStreamer, typename hdf5Real, typename TGrid>
inline void DumpHDF5(const TGrid&, const int, const double, const std::string&,
                     const std::string& = std::string("."), const bool = true) {}
