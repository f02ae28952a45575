// Host stand-in for <optix.h>, used only to compile the reference's shading
// headers on the CPU (oracle/ref_host.cpp).  The headers name one OptiX type.
#pragma once
typedef unsigned long long OptixTraversableHandle;
