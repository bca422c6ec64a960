/* A C host of the library's HDF5 reader (test infrastructure): the shape
 * and a slice of a float dataset, two elements of an integer one, and a
 * missing dataset reported through croma_b200_last_error. */
#include <stdio.h>

#include "croma_b200.h"

int main(int argc, char **argv)
{
    int rank = 0, cls = -1, size = 0;
    long long dims[4] = {0, 0, 0, 0}, ids[2] = {0, 0};
    double v[3] = {0.0, 0.0, 0.0};
    if (argc < 2) return 9;
    if (croma_b200_h5_shape(argv[1], "density", &rank, dims, 4, &cls, &size) != 0) return 1;
    if (croma_b200_h5_read_f64(argv[1], "density", 2, 3, v) != 0) return 2;
    if (croma_b200_h5_read_i64(argv[1], "particle_ID", 0, 2, ids) != 0) return 3;
    printf("%d %lld %d %d %.17g %.17g %.17g %lld %lld\n", rank, dims[0], cls, size, v[0], v[1], v[2], ids[0], ids[1]);
    if (croma_b200_h5_read_f64(argv[1], "no_such_field", 0, 1, v) == 0) return 4;
    printf("%s\n", croma_b200_last_error());
    return 0;
}
