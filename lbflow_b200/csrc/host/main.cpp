// LBFlow command line on the B200 engine: `LBFlow input.prm`.
//
// Same invocation, output files, log lines and exit contract as LBFlow's
// solver/apps/LBSim/lbsim.cpp:16-74: on any error the message is printed as
// "<rank> Failed to excute: <message>" and the process exits non-zero
// without printing "Simulation finished!".
#include <cstdlib>
#include <exception>
#include <iostream>
#include <stdexcept>

#include "prm.h"
#include "simulation.h"

using namespace lbfhost;

int main(int argc, char* argv[])
{
    const int rank = 0;
    try {
        if (argc < 2) {
            std::cerr << argv[0] << ": you must specify an input filename." << std::endl;
            return 1;
        }
        StepLog logger(std::cout);
        logger.log("Model constructing...", false);
        Params input(argv[1]);
        const std::string& model = input.fluidModel();
        if (model != "color" && model != "scsp") {
            if (model == "shanchen") {
                input.validate();
                throw std::invalid_argument("Main(): Fluid model shanchen currently not supported.");
            }
            throw std::invalid_argument("Main(): Unsupport fluid model (only color model and single components "
                                        "single phase model are supported at this time)");
        }
        Simulation sim(input);
        logger.log("Done!\n");
        logger.reset();
        logger.log("Simulation started!\n", false);
        sim.run(std::cout);
        logger.log("Simulation finished!\nTotal ");
    } catch (std::exception& e) {
        std::cout << rank << " Failed to excute: " << e.what() << std::endl;
        std::cout.flush();
        return EXIT_FAILURE;
    }
    return 0;
}
