// Name tables of the CGNS library that the reference's grid converters
// reference; the oracle never converts CGNS files, so they stay empty.
extern "C" {
const char *BCTypeName[64] = {0};
const char *PointSetTypeName[64] = {0};
}
