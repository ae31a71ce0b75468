/* Empty stand-in: the LeCo integer hot path does not use this library. */
#pragma once
