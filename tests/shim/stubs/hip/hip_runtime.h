// Stand-in for the HIP runtime header that the reference's gpu/ headers include: the B200
// shim is plain C++ over libakmc_b200.so and needs only the error type name to parse them.
#pragma once
typedef int hipError_t;
