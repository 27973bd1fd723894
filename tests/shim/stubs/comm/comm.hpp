// Stand-in for libcomm's comm/comm.hpp umbrella header: the declarations the reference uses from it are
// in the other stand-ins.
#pragma once
#include <comm/domain/colored_domain.h>
