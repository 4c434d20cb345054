// ktt_tuning_launcher -- runs a KTT JSON tuning script against this library, as KTT's
// TuningLauncher does (TuningLoader/TuningLauncher.cpp:8-56):
//
//     ktt_tuning_launcher <script.json> [NAME=VALUE ...]
//
// NAME=VALUE pairs replace "$NAME" placeholders in the script before it is read.
#include <iostream>
#include <map>
#include <string>

#include <Ktt.h>

int main(int argc, char** argv)
{
    if (argc < 2)
    {
        std::cerr << "Path to the tuning file must be specified as a command line parameter." << std::endl;
        return 1;
    }

    std::map<std::string, std::string> parameters;

    for (int i = 2; i < argc; ++i)
    {
        const std::string token = argv[i];
        const auto eq = token.find('=');

        if (eq == std::string::npos)
        {
            std::cerr << "Parameters must have the form NAME=VALUE: " << token << std::endl;
            return 1;
        }

        parameters[token.substr(0, eq)] = token.substr(eq + 1);
    }

    try
    {
        ktt::TuningLoader loader;
        loader.LoadTuningFile(argv[1], parameters);
        loader.ExecuteCommands();
    }
    catch (const std::exception& e)
    {
        std::cerr << "Error: " << e.what() << std::endl;
        return 1;
    }

    return 0;
}
