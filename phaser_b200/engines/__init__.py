"""B200 engines behind phaser's EngineHook signature `run_engine(args, props) -> state`."""
