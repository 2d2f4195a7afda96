/* Oracle build shim (test infrastructure only): intentionally empty. */
#pragma once
