// oneTBB <tbb/task.h>: nothing of it is used beyond the headers above
#pragma once

#include "tbb/task_arena.h"
#include "tbb/task_group.h"
