#pragma once

#include <helix/examples.h>
#include <helix/types.h>
