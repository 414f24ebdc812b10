// io::DataSet with the reference's constructor and accessors
// (src/io/dataset.h:13-79): a raw little-endian float32 file of
// number_of_data rows of number_of_dimensions floats.  Errors throw
// std::runtime_error instead of exit(1) (src/io/dataset.cpp:30-33).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace ursus {

typedef float Point;
typedef unsigned int ui;

enum DataSetType { DATASET_TYPE_INVALID = -1, DATASET_TYPE_BINARY = 1 };
enum DataType { DATA_TYPE_INVALID = -1, DATA_TYPE_REAL = 1, DATA_TYPE_SYNTHETIC = 2 };
enum ClusterType {
  CLUSTER_TYPE_INVALID = -1,
  CLUSTER_TYPE_NONE = 1,
  CLUSTER_TYPE_HILBERT = 2,
  CLUSTER_TYPE_KMEANSHILBERT = 3
};

namespace io {

class DataSet {
 public:
  DataSet(ui number_of_dimensions, ui number_of_data, std::string data_set_path,
          DataSetType data_set_type, DataType data_type, ClusterType cluster_type,
          std::string force_rebuild);
  // In-memory data set (no file), rows of number_of_dimensions floats.
  DataSet(ui number_of_dimensions, std::vector<Point> rows);

  ui GetNumberOfDims() const { return number_of_dimensions; }
  ui GetNumberOfData() const { return number_of_data; }
  std::string GetDataSetPath() const { return data_set_path; }
  DataSetType GetDataSetType() const { return data_set_type; }
  DataType GetDataType() const { return data_type; }
  ClusterType GetClusterType() const { return cluster_type; }
  const std::vector<Point>& GetPoints() const { return points; }
  bool IsRebuild() const { return force_rebuild == "yes"; }

 private:
  ui number_of_dimensions = 0;
  ui number_of_data = 0;
  std::string data_set_path;
  DataSetType data_set_type = DATASET_TYPE_INVALID;
  DataType data_type = DATA_TYPE_INVALID;
  ClusterType cluster_type = CLUSTER_TYPE_INVALID;
  std::vector<Point> points;
  std::string force_rebuild;
};

}  // namespace io
}  // namespace ursus
