/* Empty stand-in: the reference includes curand but its hot path does not use it. */
#pragma once
