/* Oracle test infrastructure: empty stand-in (see curand_kernel.h). */
#pragma once
