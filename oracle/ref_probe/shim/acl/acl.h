// Empty stand-in for the vendor runtime header (the probed headers need no runtime).
#pragma once
