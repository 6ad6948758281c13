// CPU ORACLE — test infrastructure. Stand-in for the HDF5 C++ header: the
// reference's SimParams3D declares methods taking H5::DataSet&, which the
// oracle never calls; a declaration of the class is all they need.
#pragma once
namespace H5 { class DataSet; }
