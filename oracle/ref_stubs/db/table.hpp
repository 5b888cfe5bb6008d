// Stand-in for the reference's include/db/table.hpp: the kernels only need
// Column (include/db/column.hpp); the catalog's DuckDB types are not used.
#pragma once
#include "db/column.hpp"
