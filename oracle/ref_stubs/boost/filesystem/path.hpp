/* Empty stand-in: the reference includes this header but the code compiled here does not use it. */
#pragma once
