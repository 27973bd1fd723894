// Stand-in for libcomm's comm/preset/sector_forwarding_region.h: the B200 shim forwards no regions.
#pragma once
#include <comm/domain/region.hpp>
