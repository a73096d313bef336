// Stand-in for sutil/Camera.h: optixScan.cpp includes it but uses nothing from it.
#pragma once
