// io/ildg.h -- ILDG configuration files (reference src/io/ildg.h:17-20): dirpath/filename/filename,
// LIME records written and read by libqcb (no c-lime, no MPI-IO).
#pragma once
#include <string>

#include "../gauge/GaugeField.h"
#include "../mpi/MpiTopology.h"

void save_ildg_clime(const std::string& filename, const std::string& dirpath, const GaugeField& field,
                     const GeometryCB& geo, const mpi::MpiTopology& topo);
void read_ildg_clime(const std::string& filename, const std::string& dirpath, GaugeField& field,
                     const GeometryCB& geo, mpi::MpiTopology& topo);
